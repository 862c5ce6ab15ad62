// Longitude (Fourier) stage: a mixed-radix (2/3/4) Stockham FFT of length
// H = nphi/2, one warp per latitude row, wrapped in the real-field
// pack/recombine that turns it into a length-nphi real transform.
//
// Conventions (fourier.ts:291-386 of the reference derives the same
// identities): with X[k] the Hermitian spectrum of a real row, X[0] = Re F_0,
// X[k] = F_k for 1 <= k <= mmax and 0 above,
//   synthesis: Z[k] = (X[k] + conj X[H-k]) + i e^{+2 pi i k/nphi} (X[k] - conj X[H-k]),
//              z = FFT_H^{+}(Z),  x[2j] = Re z[j],  x[2j+1] = Im z[j];
//   analysis:  z[j] = x[2j] + i x[2j+1],  Z = FFT_H^{-}(z),
//              X[k] = (Z[k] + conj Z[H-k])/2 - i e^{-2 pi i k/nphi} (Z[k] - conj Z[H-k])/2.
// Both unnormalised; the 2*pi/nphi of the analysis lives in the Gauss weights.
// All twiddles come from one f64-computed table tw[k] = e^{2 pi i k/nphi}.
#pragma once
#include "ts_common.cuh"

template <int SIGN>
TS_DEV float2 ts_tw(const float2 *tw, int idx) {
  const float2 w = tw[idx];
  return SIGN > 0 ? w : make_float2(w.x, -w.y);
}

// One radix-R Stockham stage: out[(t - j) R + j + q ns] = DFT_R(x_q w^{q j}),
// x_q = in[t + q H/R], j = t mod ns, w = e^{SIGN 2 pi i / (ns R)}.
template <int R, int SIGN>
TS_DEV void ts_fft_stage(const float2 *src, float2 *dst, const float2 *tw, int H, int ns,
                         int twstep, int lane) {
  const int mR = H / R;
  for (int t = lane; t < mR; t += 32) {
    const int j = t % ns;
    float2 x[R];
#pragma unroll
    for (int q = 0; q < R; q++) x[q] = src[t + q * mR];
    if (j) {
#pragma unroll
      for (int q = 1; q < R; q++) x[q] = c_mul(x[q], ts_tw<SIGN>(tw, q * j * twstep));
    }
    float2 y[R];
    if (R == 2) {
      y[0] = c_add(x[0], x[1]);
      y[1] = c_sub(x[0], x[1]);
    } else if (R == 3) {
      // y1 = x0 + w x1 + w^2 x2, w = e^{SIGN 2 pi i/3} = -1/2 + SIGN i sqrt(3)/2
      const float2 s12 = c_add(x[1], x[2]);
      const float2 d12 = c_sub(x[1], x[2]);
      const float2 mid = make_float2(x[0].x - 0.5f * s12.x, x[0].y - 0.5f * s12.y);
      const float h = SIGN * 0.8660254037844386f;
      const float2 rot = make_float2(-h * d12.y, h * d12.x);  // SIGN i sqrt3/2 (x1 - x2)
      y[0] = c_add(x[0], s12);
      y[1] = c_add(mid, rot);
      y[2] = c_sub(mid, rot);
    } else if (R == 4) {
      const float2 a = c_add(x[0], x[2]);
      const float2 b = c_sub(x[0], x[2]);
      const float2 c = c_add(x[1], x[3]);
      const float2 e = c_sub(x[1], x[3]);
      const float2 d = SIGN > 0 ? c_mul_i(e) : c_mul_negi(e);
      y[0] = c_add(a, c);
      y[1] = c_add(b, d);
      y[2] = c_sub(a, c);
      y[3] = c_sub(b, d);
    }
    const int ob = (t - j) * R + j;
#pragma unroll
    for (int q = 0; q < R; q++) dst[ob + q * ns] = y[q];
  }
}

// Full H-point FFT of the row in buffer a (b is the ping-pong partner).
// Returns the buffer holding the result.  Warp-synchronous.
template <int SIGN>
TS_DEV float2 *ts_fft_row(float2 *a, float2 *b, const float2 *tw, const TsFftTab &ft, int lane) {
  float2 *src = a, *dst = b;
  int ns = 1;
  for (int s = 0; s < ft.nst; s++) {
    const int R = ft.radix[s];
    const int twstep = ft.nphi / (ns * R);
    __syncwarp();
    if (R == 4)
      ts_fft_stage<4, SIGN>(src, dst, tw, ft.H, ns, twstep, lane);
    else if (R == 2)
      ts_fft_stage<2, SIGN>(src, dst, tw, ft.H, ns, twstep, lane);
    else
      ts_fft_stage<3, SIGN>(src, dst, tw, ft.H, ns, twstep, lane);
    float2 *tmp = src;
    src = dst;
    dst = tmp;
    ns *= R;
  }
  __syncwarp();
  return src;
}

// X[k] of the Hermitian spectrum from a staged column (tile[k*LB + w]).
TS_DEV float2 ts_spec_at(const float2 *tile, int LB, int w, int k, int mmax) {
  if (k == 0) return make_float2(tile[w].x, 0.f);
  if (k <= mmax) return tile[k * LB + w];
  return make_float2(0.f, 0.f);
}

// Build Z (the packed half-length spectrum) for the synthesis of one row.
TS_DEV void ts_pack_synth(float2 *row, const float2 *tile, int LB, int w, const float2 *tw,
                          const TsFftTab &ft, int lane) {
  const int H = ft.H;
  for (int k = lane; k < H; k += 32) {
    const float2 xk = ts_spec_at(tile, LB, w, k, ft.mmax);
    const float2 cj = c_conj(ts_spec_at(tile, LB, w, H - k, ft.mmax));
    const float2 b = c_mul(c_sub(xk, cj), tw[k]);
    row[k] = c_add(c_add(xk, cj), c_mul_i(b));
  }
}

// Recombine the forward FFT of a packed row into X[k], k <= mmax, written to
// tile[k*LB + w].
TS_DEV void ts_unpack_analys(const float2 *Z, float2 *tile, int LB, int w, const float2 *tw,
                             const TsFftTab &ft, int lane) {
  const int H = ft.H;
  for (int k = lane; k <= ft.mmax; k += 32) {
    const float2 zk = Z[k];
    const float2 zh = c_conj(Z[k == 0 ? 0 : H - k]);
    const float2 xe = c_scale(c_add(zk, zh), 0.5f);
    const float2 xo = c_mul_negi(c_scale(c_sub(zk, zh), 0.5f));
    tile[k * LB + w] = c_add(xe, c_mul(xo, ts_tw<-1>(tw, k)));
  }
}

// Shared-memory carve-up of a Fourier CTA with LB rows (one warp each):
//   tw[nphi] | tile[(mmax+1)*LB] | rows[LB][nbuf][H]
TS_DEV float2 *ts_four_tw(float2 *smem) { return smem; }
TS_DEV float2 *ts_four_tile(float2 *smem, const TsFftTab &ft) { return smem + ft.nphi; }
TS_DEV float2 *ts_four_rows(float2 *smem, const TsFftTab &ft, int LB) {
  return smem + ft.nphi + (ft.mmax + 1) * LB;
}

TS_DEV void ts_load_tw(float2 *stw, const TsFftTab &ft) {
  for (int i = threadIdx.x; i < ft.nphi; i += blockDim.x) stw[i] = ft.tw[i];
}

// Stage the (mmax+1) x LB block fm[m][lat0..lat0+LB) of one field.
TS_DEV void ts_load_tile(float2 *tile, const float2 *src, int lat0, int LB, const TsFftTab &ft) {
  const int n = (ft.mmax + 1) * LB;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int k = idx / LB, w = idx - k * LB;
    const int lat = lat0 + w;
    tile[idx] = lat < ft.nlat ? src[(long)k * ft.nlat + lat] : make_float2(0.f, 0.f);
  }
}

TS_DEV void ts_store_tile(const float2 *tile, float2 *dst, int lat0, int LB, const TsFftTab &ft) {
  const int n = (ft.mmax + 1) * LB;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int k = idx / LB, w = idx - k * LB;
    const int lat = lat0 + w;
    if (lat < ft.nlat) dst[(long)k * ft.nlat + lat] = tile[idx];
  }
}

// fm[field][m][lat] -> spat[field][lat][phi].  grid = (ceil(nlat/LB), nfields),
// block = 32*LB threads.
__global__ void __launch_bounds__(512)
ts_fourier_synth(TsFftTab ft, const float2 *__restrict__ fm, long fm_stride,
                 float *__restrict__ spat, long spat_stride) {
  extern __shared__ float2 ts_smem_fs[];
  const int LB = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * LB;
  const long f = blockIdx.y;
  float2 *stw = ts_four_tw(ts_smem_fs);
  float2 *tile = ts_four_tile(ts_smem_fs, ft);
  float2 *rows = ts_four_rows(ts_smem_fs, ft, LB) + (long)w * 2 * ft.H;
  ts_load_tw(stw, ft);
  ts_load_tile(tile, fm + f * fm_stride, lat0, LB, ft);
  __syncthreads();
  const int lat = lat0 + w;
  if (lat >= ft.nlat) return;
  ts_pack_synth(rows, tile, LB, w, stw, ft, lane);
  const float2 *z = ts_fft_row<+1>(rows, rows + ft.H, stw, ft, lane);
  float2 *out = reinterpret_cast<float2 *>(spat + f * spat_stride + (long)lat * ft.nphi);
  for (int j = lane; j < ft.H; j += 32) out[j] = z[j];
}

// spat[field][lat][phi] -> g[field][m][lat] (unnormalised).
__global__ void __launch_bounds__(512)
ts_fourier_analys(TsFftTab ft, const float *__restrict__ spat, long spat_stride,
                  float2 *__restrict__ g, long g_stride) {
  extern __shared__ float2 ts_smem_fa[];
  const int LB = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * LB;
  const long f = blockIdx.y;
  float2 *stw = ts_four_tw(ts_smem_fa);
  float2 *tile = ts_four_tile(ts_smem_fa, ft);
  float2 *rows = ts_four_rows(ts_smem_fa, ft, LB) + (long)w * 2 * ft.H;
  ts_load_tw(stw, ft);
  __syncthreads();
  const int lat = lat0 + w;
  if (lat < ft.nlat) {
    const float2 *in = reinterpret_cast<const float2 *>(spat + f * spat_stride + (long)lat * ft.nphi);
    for (int j = lane; j < ft.H; j += 32) rows[j] = in[j];
    const float2 *Z = ts_fft_row<-1>(rows, rows + ft.H, stw, ft, lane);
    ts_unpack_analys(Z, tile, LB, w, stw, ft, lane);
  }
  __syncthreads();
  ts_store_tile(tile, g + f * g_stride, lat0, LB, ft);
}

// ------------------------------------------------------- fused grid phase
//
// One launch runs a whole grid phase of a compiled model for a block of LB
// latitude rows of one instance: the synthesis FFTs of the phase's NSYN
// spectral inputs, the generated element-wise program at every grid point
// (Prog::eval: reaction terms and any other grid statement), and the analysis
// FFTs of its NANA outputs.  The grid values live in shared memory and
// registers only; a grid variable reaches HBM only when it is materialised
// (NGOUT outputs: a displayed field, or a value a later phase reads).
//
//   fm [inst][NSYN][mmax+1][nlat]   -> rows -> eval -> rows -> gm [inst][NANA][mmax+1][nlat]


template <class Prog>
__global__ void __launch_bounds__(512) ts_fourier_phase(TsFftTab ft, TsPhaseIO io) {
  constexpr int NSYN = Prog::NSYN, NGIN = Prog::NGIN, NANA = Prog::NANA, NGOUT = Prog::NGOUT;
  constexpr int NR = NSYN + NANA + 1;  // rows per warp: inputs, outputs, one ping-pong row
  extern __shared__ float2 ts_smem_fp[];
  const int LB = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * LB;
  const long inst = blockIdx.y;
  const int lat = lat0 + w;
  const bool live = lat < ft.nlat;
  float2 *stw = ts_four_tw(ts_smem_fp);
  float2 *tile = ts_four_tile(ts_smem_fp, ft);
  float2 *rowbase = ts_four_rows(ts_smem_fp, ft, LB) + (long)w * NR * ft.H;
  float2 *rp[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) rp[r] = rowbase + (long)r * ft.H;
  ts_load_tw(stw, ft);

  // synthesis of every spectral input of the phase
#pragma unroll
  for (int s = 0; s < NSYN; s++) {
    __syncthreads();
    ts_load_tile(tile, io.fm + (inst * NSYN + s) * io.field, lat0, LB, ft);
    __syncthreads();
    if (live) {
      ts_pack_synth(rp[s], tile, LB, w, stw, ft, lane);
      const float2 *z = ts_fft_row<+1>(rp[s], rp[NR - 1], stw, ft, lane);
      if (z != rp[s]) {
        float2 *tmp = rp[s];
        rp[s] = rp[NR - 1];
        rp[NR - 1] = tmp;
      }
    }
  }

  // the element-wise program, two grid points (one packed complex) at a time
  if (live) {
    const float *prm = io.prm + inst * io.nprm;
    const long rowoff = (long)lat * ft.nphi;
    for (int j = lane; j < ft.H; j += 32) {
      float in0[NSYN + NGIN > 0 ? NSYN + NGIN : 1], in1[NSYN + NGIN > 0 ? NSYN + NGIN : 1];
#pragma unroll
      for (int s = 0; s < NSYN; s++) {
        const float2 z = rp[s][j];
        in0[s] = z.x;
        in1[s] = z.y;
      }
#pragma unroll
      for (int gi = 0; gi < NGIN; gi++) {
        const float2 x = *reinterpret_cast<const float2 *>(io.gin[gi] + inst * io.gin_stride[gi] +
                                                           rowoff + 2 * j);
        in0[NSYN + gi] = x.x;
        in1[NSYN + gi] = x.y;
      }
      float out0[NANA + NGOUT > 0 ? NANA + NGOUT : 1], out1[NANA + NGOUT > 0 ? NANA + NGOUT : 1];
      Prog::eval(in0, out0, prm);
      Prog::eval(in1, out1, prm);
#pragma unroll
      for (int k = 0; k < NANA; k++) rp[NSYN + k][j] = make_float2(out0[k], out1[k]);
#pragma unroll
      for (int o = 0; o < NGOUT; o++)
        *reinterpret_cast<float2 *>(io.gout[o] + inst * io.gout_stride[o] + rowoff + 2 * j) =
            make_float2(out0[NANA + o], out1[NANA + o]);
    }
  }

  // analysis of every output of the phase
#pragma unroll
  for (int k = 0; k < NANA; k++) {
    if (live) {
      const float2 *Z = ts_fft_row<-1>(rp[NSYN + k], rp[NR - 1], stw, ft, lane);
      if (Z != rp[NSYN + k]) {
        float2 *tmp = rp[NSYN + k];
        rp[NSYN + k] = rp[NR - 1];
        rp[NR - 1] = tmp;
      }
      ts_unpack_analys(rp[NSYN + k], tile, LB, w, stw, ft, lane);
    }
    __syncthreads();
    ts_store_tile(tile, io.gm + (inst * NANA + k) * io.field, lat0, LB, ft);
    __syncthreads();
  }
}

// ====================================================== warp-register FFT
//
// For H = R1 * 32 (R1 <= 24) a row lives in registers: lane t, register j
// holds element n = t + 32 j ("natural" layout).  The transform is split as
//   X[k1 + R1 k2] = sum_t w32^{t k2} [ wH^{t k1} sum_j x[t + 32 j] wR1^{j k1} ]
// into an R1-point DFT inside each lane, a per-lane twiddle, and a 32-point
// transform across the lanes done with shuffles.  With decimation in
// frequency across the lanes (ts_fft_dif) the result lands "permuted": lane
// t, register k1 holds k = k1 + R1 rev5(t).  The decimation-in-time form
// (ts_fft_dit) is the exact inverse sequence: permuted in, natural out.  A
// synthesis (DIF, sign +) followed by an analysis (DIT, sign -) therefore
// never needs the row in natural order in between, which is what lets the
// fused model phase evaluate the reaction point by point in registers.

template <int M>
struct TsRadix {
  static constexpr int value = (M % 4 == 0) ? 4 : (M % 2 == 0) ? 2 : 3;
};

template <int R, int SIGN>
TS_DEV void ts_butterfly(float2 (&a)[R]) {
  if constexpr (R == 2) {
    const float2 s = c_add(a[0], a[1]), d = c_sub(a[0], a[1]);
    a[0] = s;
    a[1] = d;
  } else if constexpr (R == 3) {
    const float2 s12 = c_add(a[1], a[2]);
    const float2 d12 = c_sub(a[1], a[2]);
    const float2 mid = make_float2(a[0].x - 0.5f * s12.x, a[0].y - 0.5f * s12.y);
    const float h = SIGN * 0.8660254037844386f;
    const float2 rot = make_float2(-h * d12.y, h * d12.x);
    a[0] = c_add(a[0], s12);
    a[1] = c_add(mid, rot);
    a[2] = c_sub(mid, rot);
  } else if constexpr (R == 4) {
    const float2 p = c_add(a[0], a[2]), q = c_sub(a[0], a[2]);
    const float2 r = c_add(a[1], a[3]), e = c_sub(a[1], a[3]);
    const float2 d = SIGN > 0 ? c_mul_i(e) : c_mul_negi(e);
    a[0] = c_add(p, r);
    a[1] = c_add(q, d);
    a[2] = c_sub(p, r);
    a[3] = c_sub(q, d);
  }
}

// N-point DFT (sign SIGN) of a register array, natural order in and out:
// Stockham stages with compile-time radices; twiddles from the shared table
// tw[k] = e^{2 pi i k/nphi} (uniform across lanes).
template <int N, int NS, int SIGN>
TS_DEV void ts_reg_dft(float2 (&x)[N], const float2 *tw, int nphi) {
  if constexpr (NS < N) {
    constexpr int R = TsRadix<N / NS>::value;
    constexpr int MR = N / R;
    float2 y[N];
    const int twstep = nphi / (NS * R);
#pragma unroll
    for (int t = 0; t < MR; t++) {
      const int j = t % NS;
      float2 a[R];
#pragma unroll
      for (int q = 0; q < R; q++) a[q] = x[t + q * MR];
      if (j) {
#pragma unroll
        for (int q = 1; q < R; q++) a[q] = c_mul(a[q], ts_tw<SIGN>(tw, q * j * twstep));
      }
      ts_butterfly<R, SIGN>(a);
#pragma unroll
      for (int q = 0; q < R; q++) y[(t - j) * R + j + q * NS] = a[q];
    }
#pragma unroll
    for (int i = 0; i < N; i++) x[i] = y[i];
    ts_reg_dft<N, NS * R, SIGN>(x, tw, nphi);
  }
}

// Per-lane constants of the cross-lane stages: w5[s] = e^{+2 pi i (t mod h)/(2h)},
// h = 16 >> s.
TS_DEV void ts_lane_twiddles(float2 (&w5)[5], const float2 *tw, int nphi, int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int h = 16 >> s;
    w5[s] = tw[(lane & (h - 1)) * (nphi / (2 * h))];
  }
}

// twr[k1*32 + t] = e^{+2 pi i t k1 / H} (H = nphi/2): the per-lane twiddles
TS_DEV void ts_load_twr(float2 *twr, const float2 *tw, int R1, int nphi) {
  for (int i = threadIdx.x; i < R1 * 32; i += blockDim.x) {
    const int k1 = i >> 5, t = i & 31;
    twr[i] = tw[(2 * t * k1) % nphi];
  }
}

TS_DEV float2 ts_shfl_xor2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

template <int R1, int SIGN>
TS_DEV void ts_fft_dif(float2 (&x)[R1], const float2 *tw, const float2 *twr,
                       const float2 (&w5)[5], int nphi, int lane) {
  ts_reg_dft<R1, 1, SIGN>(x, tw, nphi);
#pragma unroll
  for (int k1 = 1; k1 < R1; k1++) {
    const float2 w = twr[k1 * 32 + lane];
    x[k1] = c_mul(x[k1], SIGN > 0 ? w : c_conj(w));
  }
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int h = 16 >> s;
    const bool upper = (lane & h) != 0;
    const float2 w = SIGN > 0 ? w5[s] : c_conj(w5[s]);
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) {
      const float2 p = ts_shfl_xor2(x[k1], h);
      x[k1] = upper ? c_mul(c_sub(p, x[k1]), w) : c_add(x[k1], p);
    }
  }
}

template <int R1, int SIGN>
TS_DEV void ts_fft_dit(float2 (&x)[R1], const float2 *tw, const float2 *twr,
                       const float2 (&w5)[5], int nphi, int lane) {
#pragma unroll
  for (int s = 4; s >= 0; s--) {
    const int h = 16 >> s;
    const bool upper = (lane & h) != 0;
    const float2 w = SIGN > 0 ? w5[s] : c_conj(w5[s]);
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) {
      const float2 own = upper ? c_mul(x[k1], w) : x[k1];
      const float2 p = ts_shfl_xor2(own, h);
      x[k1] = upper ? c_sub(p, own) : c_add(own, p);
    }
  }
#pragma unroll
  for (int k1 = 1; k1 < R1; k1++) {
    const float2 w = twr[k1 * 32 + lane];
    x[k1] = c_mul(x[k1], SIGN > 0 ? w : c_conj(w));
  }
  ts_reg_dft<R1, 1, SIGN>(x, tw, nphi);
}

TS_DEV int ts_rev5(int t) { return __brev((unsigned)t) >> 27; }

// Shared-memory carve-up of a register-FFT CTA with LB rows:
//   tw[nphi] | twr[H] | tile[LB][P], P = mmax + 2 | rowbuf[LB][H]
TS_DEV int ts_rtile_pitch(const TsFftTab &ft) { return ft.mmax + 2; }

// X[k] (Hermitian spectrum) of row w from a [w][k] tile
TS_DEV float2 ts_rspec(const float2 *trow, int k, int mmax) {
  if (k == 0) return make_float2(trow[0].x, 0.f);
  if (k <= mmax) return trow[k];
  return make_float2(0.f, 0.f);
}

// stage fm[m][lat0..lat0+LB) of one field into tile[w][k] (coalesced reads)
TS_DEV void ts_load_rtile(float2 *tile, const float2 *src, int lat0, int LB, const TsFftTab &ft) {
  const int P = ts_rtile_pitch(ft);
  const int n = (ft.mmax + 1) * LB;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int k = idx / LB, w = idx - k * LB;
    const int lat = lat0 + w;
    tile[w * P + k] = lat < ft.nlat ? src[(long)k * ft.nlat + lat] : make_float2(0.f, 0.f);
  }
}

TS_DEV void ts_store_rtile(const float2 *tile, float2 *dst, int lat0, int LB, const TsFftTab &ft) {
  const int P = ts_rtile_pitch(ft);
  const int n = (ft.mmax + 1) * LB;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int k = idx / LB, w = idx - k * LB;
    const int lat = lat0 + w;
    if (lat < ft.nlat) dst[(long)k * ft.nlat + lat] = tile[w * P + k];
  }
}

// Z[n] of the packed half-length synthesis input, lane-natural layout
template <int R1>
TS_DEV void ts_rpack(float2 (&x)[R1], const float2 *trow, const float2 *tw, const TsFftTab &ft,
                     int lane) {
  const int H = ft.H;
#pragma unroll
  for (int j = 0; j < R1; j++) {
    const int k = lane + 32 * j;
    const float2 xk = ts_rspec(trow, k, ft.mmax);
    const float2 cj = c_conj(ts_rspec(trow, H - k, ft.mmax));
    x[j] = c_add(c_add(xk, cj), c_mul_i(c_mul(c_sub(xk, cj), tw[k])));
  }
}

// analysis recombination from a row of Z in natural order (zrow[k]) into trow[k]
TS_DEV void ts_runpack(const float2 *zrow, float2 *trow, const float2 *tw, const TsFftTab &ft,
                       int lane) {
  const int H = ft.H;
  for (int k = lane; k <= ft.mmax; k += 32) {
    const float2 zk = zrow[k];
    const float2 zh = c_conj(zrow[k == 0 ? 0 : H - k]);
    const float2 xe = c_scale(c_add(zk, zh), 0.5f);
    const float2 xo = c_mul_negi(c_scale(c_sub(zk, zh), 0.5f));
    trow[k] = c_add(xe, c_mul(xo, ts_tw<-1>(tw, k)));
  }
}

TS_DEV size_t ts_rfft_smem_floats2(const TsFftTab &ft, int LB, int nrowbuf) {
  return (size_t)ft.nphi + ft.H + (size_t)LB * ts_rtile_pitch(ft) + (size_t)LB * nrowbuf * ft.H;
}

// fm[field][m][lat] -> spat[field][lat][phi], register FFT.  grid =
// (ceil(nlat/LB), nfields), block = 32*LB.
template <int R1>
__global__ void __launch_bounds__(256)
ts_fourier_synth_r(TsFftTab ft, const float2 *__restrict__ fm, long fm_stride,
                   float *__restrict__ spat, long spat_stride) {
  extern __shared__ float2 ts_smem_rs[];
  const int LB = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * LB;
  const long f = blockIdx.y;
  const int P = ts_rtile_pitch(ft);
  float2 *stw = ts_smem_rs;
  float2 *twr = stw + ft.nphi;
  float2 *tile = twr + ft.H;
  float2 *rowbuf = tile + LB * P + (long)w * ft.H;
  ts_load_tw(stw, ft);
  __syncthreads();
  ts_load_twr(twr, stw, R1, ft.nphi);
  ts_load_rtile(tile, fm + f * fm_stride, lat0, LB, ft);
  __syncthreads();
  const int lat = lat0 + w;
  if (lat >= ft.nlat) return;
  float2 w5[5];
  ts_lane_twiddles(w5, stw, ft.nphi, lane);
  float2 x[R1];
  ts_rpack<R1>(x, tile + w * P, stw, ft, lane);
  ts_fft_dif<R1, +1>(x, stw, twr, w5, ft.nphi, lane);
  // permuted (lane, k1) -> rowbuf[k1*32 + lane]; read back in natural order
#pragma unroll
  for (int k1 = 0; k1 < R1; k1++) rowbuf[k1 * 32 + lane] = x[k1];
  __syncwarp();
  float2 *out = reinterpret_cast<float2 *>(spat + f * spat_stride + (long)lat * ft.nphi);
  for (int n = lane; n < ft.H; n += 32) {
    const int k1 = n % R1, k2 = n / R1;
    out[n] = rowbuf[k1 * 32 + ts_rev5(k2)];
  }
}

// spat[field][lat][phi] -> g[field][m][lat], register FFT.
template <int R1>
__global__ void __launch_bounds__(256)
ts_fourier_analys_r(TsFftTab ft, const float *__restrict__ spat, long spat_stride,
                    float2 *__restrict__ g, long g_stride) {
  extern __shared__ float2 ts_smem_ra[];
  const int LB = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * LB;
  const long f = blockIdx.y;
  const int P = ts_rtile_pitch(ft);
  float2 *stw = ts_smem_ra;
  float2 *twr = stw + ft.nphi;
  float2 *tile = twr + ft.H;
  float2 *rowbuf = tile + LB * P + (long)w * ft.H;
  ts_load_tw(stw, ft);
  __syncthreads();
  ts_load_twr(twr, stw, R1, ft.nphi);
  __syncthreads();
  const int lat = lat0 + w;
  if (lat < ft.nlat) {
    float2 w5[5];
    ts_lane_twiddles(w5, stw, ft.nphi, lane);
    const float2 *in = reinterpret_cast<const float2 *>(spat + f * spat_stride + (long)lat * ft.nphi);
    float2 x[R1];
#pragma unroll
    for (int j = 0; j < R1; j++) x[j] = in[lane + 32 * j];
    ts_fft_dif<R1, -1>(x, stw, twr, w5, ft.nphi, lane);
    // permuted -> natural order in rowbuf, then recombine
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) rowbuf[k1 + R1 * ts_rev5(lane)] = x[k1];
    __syncwarp();
    ts_runpack(rowbuf, tile + w * P, stw, ft, lane);
  }
  __syncthreads();
  ts_store_rtile(tile, g + f * g_stride, lat0, LB, ft);
}

// Fused model phase on the register FFT (see ts_fourier_phase).  The grid
// values stay in the permuted layout between the synthesis (DIF) and the
// analysis (DIT); grid inputs and materialised outputs go through rowbuf so
// that their global accesses stay coalesced.
template <class Prog, int R1>
__global__ void __launch_bounds__(256) ts_fourier_phase_r(TsFftTab ft, TsPhaseIO io) {
  constexpr int NSYN = Prog::NSYN, NGIN = Prog::NGIN, NANA = Prog::NANA, NGOUT = Prog::NGOUT;
  constexpr int NIN = NSYN + NGIN > 0 ? NSYN + NGIN : 1;
  constexpr int NOUT = NANA + NGOUT > 0 ? NANA + NGOUT : 1;
  extern __shared__ float2 ts_smem_rp[];
  const int LB = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * LB;
  const long inst = blockIdx.y;
  const int lat = lat0 + w;
  const bool live = lat < ft.nlat;
  const int P = ts_rtile_pitch(ft);
  float2 *stw = ts_smem_rp;
  float2 *twr = stw + ft.nphi;
  float2 *tile = twr + ft.H;
  float2 *rowbuf = tile + LB * P + (long)w * ft.H;
  ts_load_tw(stw, ft);
  __syncthreads();
  ts_load_twr(twr, stw, R1, ft.nphi);
  __syncthreads();
  float2 w5[5];
  ts_lane_twiddles(w5, stw, ft.nphi, lane);
  const long rowoff = (long)lat * ft.nphi;

  // grid values of every input, permuted layout: v[i][k1] = (x[2n], x[2n+1]),
  // n = k1 + R1 rev5(lane)
  float2 v[NIN][R1];
#pragma unroll
  for (int s = 0; s < NSYN; s++) {
    __syncthreads();
    ts_load_rtile(tile, io.fm + (inst * NSYN + s) * io.field, lat0, LB, ft);
    __syncthreads();
    if (live) {
      ts_rpack<R1>(v[s], tile + w * P, stw, ft, lane);
      ts_fft_dif<R1, +1>(v[s], stw, twr, w5, ft.nphi, lane);
    }
  }
#pragma unroll
  for (int gi = 0; gi < NGIN; gi++) {
    if (live) {
      const float2 *src = reinterpret_cast<const float2 *>(io.gin[gi] + inst * io.gin_stride[gi] + rowoff);
      __syncwarp();
      for (int n = lane; n < ft.H; n += 32) rowbuf[n] = src[n];
      __syncwarp();
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) v[NSYN + gi][k1] = rowbuf[k1 + R1 * ts_rev5(lane)];
    }
  }
  // the element-wise program, point by point
  float2 r[NOUT][R1];
  if (live) {
    const float *prm = io.prm + inst * io.nprm;
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) {
      float in0[NIN], in1[NIN], o0[NOUT], o1[NOUT];
#pragma unroll
      for (int i = 0; i < NSYN + NGIN; i++) {
        in0[i] = v[i][k1].x;
        in1[i] = v[i][k1].y;
      }
      Prog::eval(in0, o0, prm);
      Prog::eval(in1, o1, prm);
#pragma unroll
      for (int o = 0; o < NANA + NGOUT; o++) r[o][k1] = make_float2(o0[o], o1[o]);
    }
  }
#pragma unroll
  for (int o = 0; o < NGOUT; o++) {
    if (live) {
      __syncwarp();
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) rowbuf[k1 + R1 * ts_rev5(lane)] = r[NANA + o][k1];
      __syncwarp();
      float2 *dst = reinterpret_cast<float2 *>(io.gout[o] + inst * io.gout_stride[o] + rowoff);
      for (int n = lane; n < ft.H; n += 32) dst[n] = rowbuf[n];
    }
  }
  // analysis of every output: DIT takes the permuted layout as it is
#pragma unroll
  for (int k = 0; k < NANA; k++) {
    if (live) {
      ts_fft_dit<R1, -1>(r[k], stw, twr, w5, ft.nphi, lane);
      __syncwarp();
#pragma unroll
      for (int j = 0; j < R1; j++) rowbuf[lane + 32 * j] = r[k][j];
      __syncwarp();
      ts_runpack(rowbuf, tile + w * P, stw, ft, lane);
    }
    __syncthreads();
    ts_store_rtile(tile, io.gm + (inst * NANA + k) * io.field, lat0, LB, ft);
    __syncthreads();
  }
}

// ------------------------------------------ analysis into the TC operand image
//
// Tensor-core plans consume the analysis as W_par = w (G_north +- G_south)
// in the MMA's byte image (TsTcImg.w).  A CTA therefore takes NP northern
// latitudes and their southern mirrors (warp w: rows lat0+w and
// nlat-1-lat0-w) and writes the folded, weighted values straight into the
// image: 32-byte runs of 8 latitudes per (m, parity, re|im).
TS_DEV void ts_write_wimg(const float2 *tN, const float2 *tS, int P, int NP, int lat0, long f,
                          const TsFftTab &ft, const float *wq, char *wimg, int nfb, int fpb,
                          int nlc, int nh) {
  const long fb = f / fpb;
  const int fl = (int)(f - fb * fpb);
  const int n = (ft.mmax + 1) * 4 * NP;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int w = idx % NP;
    const int rest = idx / NP;
    const int comp = rest & 1, par = (rest >> 1) & 1, m = rest >> 2;
    const int lat = lat0 + w;
    if (lat >= nh) continue;
    const float2 xn = tN[w * P + m], xs = tS[w * P + m];
    const float a = comp ? xn.y : xn.x, b = comp ? xs.y : xs.x;
    const float v = wq[lat] * (par ? a - b : a + b);
    const long blk = (((long)m * nfb + fb) * 2 + par) * nlc + (lat >> 5);
    *reinterpret_cast<float *>(wimg + blk * 16384 + ts_swz_img(2 * fl + comp, lat & 31)) = v;
  }
}

// spat[field][lat][phi] -> W image.  grid = (ceil(nh/NP), nfields), block = 32*NP.
// Shared memory: tw[nphi] | twr[H] | tileN[NP][P] | tileS[NP][P] | rowbuf[NP][H].
template <int R1>
__global__ void __launch_bounds__(256)
ts_fourier_analys_rw(TsFftTab ft, const float *__restrict__ spat, long spat_stride,
                     const float *__restrict__ wq, char *wimg, int nfb, int fpb, int nlc, int nh) {
  extern __shared__ float2 ts_smem_rw[];
  const int NP = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * NP;
  const long f = blockIdx.y;
  const int P = ts_rtile_pitch(ft);
  float2 *stw = ts_smem_rw;
  float2 *twr = stw + ft.nphi;
  float2 *tN = twr + ft.H;
  float2 *tS = tN + NP * P;
  float2 *rowbuf = tS + NP * P + (long)w * ft.H;
  ts_load_tw(stw, ft);
  __syncthreads();
  ts_load_twr(twr, stw, R1, ft.nphi);
  __syncthreads();
  const int latN = lat0 + w;
  if (latN < nh) {
    float2 w5[5];
    ts_lane_twiddles(w5, stw, ft.nphi, lane);
    const int latS = ft.nlat - 1 - latN;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      float2 *trow = (h ? tS : tN) + w * P;
      if (h && latS == latN) {  // the equator counts once
        for (int k = lane; k <= ft.mmax; k += 32) trow[k] = make_float2(0.f, 0.f);
        continue;
      }
      const float2 *in = reinterpret_cast<const float2 *>(spat + f * spat_stride +
                                                          (long)(h ? latS : latN) * ft.nphi);
      float2 x[R1];
#pragma unroll
      for (int j = 0; j < R1; j++) x[j] = in[lane + 32 * j];
      ts_fft_dif<R1, -1>(x, stw, twr, w5, ft.nphi, lane);
      __syncwarp();
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) rowbuf[k1 + R1 * ts_rev5(lane)] = x[k1];
      __syncwarp();
      ts_runpack(rowbuf, trow, stw, ft, lane);
      __syncwarp();
    }
  }
  __syncthreads();
  ts_write_wimg(tN, tS, P, NP, lat0, f, ft, wq, wimg, nfb, fpb, nlc, nh);
}

// stage fm[m][lat] of northern (h = 0) or mirrored southern (h = 1) rows of
// the CTA's latitude pairs into tile[w][k]
TS_DEV void ts_load_rtile_pairs(float2 *tile, const float2 *src, int lat0, int NP, int h,
                                int nh, const TsFftTab &ft) {
  const int P = ts_rtile_pitch(ft);
  const int n = (ft.mmax + 1) * NP;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int k = idx / NP, w = idx - k * NP;
    const int latN = lat0 + w;
    const int lat = h ? ft.nlat - 1 - latN : latN;
    tile[w * P + k] = latN < nh ? src[(long)k * ft.nlat + lat] : make_float2(0.f, 0.f);
  }
}

// Fused model phase for tensor-core plans: as ts_fourier_phase_r, but over
// north/south latitude pairs, with the analysis outputs written as the W image
// the tensor-core analysis reads.  grid = (ceil(nh/NP), instances), block =
// 32*NP.  Shared memory: tw | twr | tin[NP][P] | tout[2][NANA][NP][P] |
// rowbuf[NP][H].
template <class Prog, int R1>
__global__ void __launch_bounds__(256) ts_fourier_phase_rw(TsFftTab ft, TsPhaseIO io) {
  constexpr int NSYN = Prog::NSYN, NGIN = Prog::NGIN, NANA = Prog::NANA, NGOUT = Prog::NGOUT;
  constexpr int NIN = NSYN + NGIN > 0 ? NSYN + NGIN : 1;
  constexpr int NOUT = NANA + NGOUT > 0 ? NANA + NGOUT : 1;
  constexpr int NA = NANA > 0 ? NANA : 1;
  extern __shared__ float2 ts_smem_rpw[];
  const int NP = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lat0 = blockIdx.x * NP;
  const long inst = blockIdx.y;
  const int P = ts_rtile_pitch(ft);
  float2 *stw = ts_smem_rpw;
  float2 *twr = stw + ft.nphi;
  float2 *tin = twr + ft.H;
  float2 *tout = tin + NP * P;  // [h][k][w][P]
  float2 *rowbuf = tout + 2 * NA * NP * P + (long)w * ft.H;
  ts_load_tw(stw, ft);
  __syncthreads();
  ts_load_twr(twr, stw, R1, ft.nphi);
  __syncthreads();
  float2 w5[5];
  ts_lane_twiddles(w5, stw, ft.nphi, lane);
  const int latN = lat0 + w;
  const float *prm = io.prm + inst * io.nprm;

#pragma unroll 1
  for (int h = 0; h < 2; h++) {
    const int lat = h ? ft.nlat - 1 - latN : latN;
    const bool equator_south = h && lat == latN;
    const bool live = latN < io.nh && !equator_south;
    const long rowoff = (long)lat * ft.nphi;
    float2 v[NIN][R1];
#pragma unroll
    for (int s = 0; s < NSYN; s++) {
      __syncthreads();
      ts_load_rtile_pairs(tin, io.fm + (inst * NSYN + s) * io.field, lat0, NP, h, io.nh, ft);
      __syncthreads();
      if (live) {
        ts_rpack<R1>(v[s], tin + w * P, stw, ft, lane);
        ts_fft_dif<R1, +1>(v[s], stw, twr, w5, ft.nphi, lane);
      }
    }
#pragma unroll
    for (int gi = 0; gi < NGIN; gi++) {
      if (live) {
        const float2 *src = reinterpret_cast<const float2 *>(io.gin[gi] + inst * io.gin_stride[gi] + rowoff);
        __syncwarp();
        for (int n = lane; n < ft.H; n += 32) rowbuf[n] = src[n];
        __syncwarp();
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) v[NSYN + gi][k1] = rowbuf[k1 + R1 * ts_rev5(lane)];
      }
    }
    float2 r[NOUT][R1];
    if (live) {
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) {
        float in0[NIN], in1[NIN], o0[NOUT], o1[NOUT];
#pragma unroll
        for (int i = 0; i < NSYN + NGIN; i++) {
          in0[i] = v[i][k1].x;
          in1[i] = v[i][k1].y;
        }
        Prog::eval(in0, o0, prm);
        Prog::eval(in1, o1, prm);
#pragma unroll
        for (int o = 0; o < NANA + NGOUT; o++) r[o][k1] = make_float2(o0[o], o1[o]);
      }
#pragma unroll
      for (int o = 0; o < NGOUT; o++) {
        __syncwarp();
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) rowbuf[k1 + R1 * ts_rev5(lane)] = r[NANA + o][k1];
        __syncwarp();
        float2 *dst = reinterpret_cast<float2 *>(io.gout[o] + inst * io.gout_stride[o] + rowoff);
        for (int n = lane; n < ft.H; n += 32) dst[n] = rowbuf[n];
      }
    }
#pragma unroll
    for (int k = 0; k < NANA; k++) {
      float2 *trow = tout + ((long)(h * NA + k) * NP + w) * P;
      if (live) {
        ts_fft_dit<R1, -1>(r[k], stw, twr, w5, ft.nphi, lane);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < R1; j++) rowbuf[lane + 32 * j] = r[k][j];
        __syncwarp();
        ts_runpack(rowbuf, trow, stw, ft, lane);
        __syncwarp();
      } else if (equator_south) {
        for (int kk = lane; kk <= ft.mmax; kk += 32) trow[kk] = make_float2(0.f, 0.f);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NANA; k++)
    ts_write_wimg(tout + (long)k * NP * P, tout + (long)(NA + k) * NP * P, P, NP, lat0,
                  inst * NANA + k, ft, io.wq, io.wimg, io.w_nfb, io.w_fpb, io.w_nlc, io.nh);
}
