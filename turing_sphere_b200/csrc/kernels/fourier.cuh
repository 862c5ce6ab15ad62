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
