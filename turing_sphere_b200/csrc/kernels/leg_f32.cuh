// Plain FP32 Legendre stage: on-the-fly three-term recurrence over l, with the
// even/odd (north/south) symmetry folded in and the recurrence coefficients and
// coefficients staged in shared memory.
//
// Synthesis (leg.ts:43-137 of the reference computes the same sum):
//   F_m(theta_i) = sum_{l=m..lmax} Q_lm ytilde_l^m(theta_i)
// Analysis (leg.ts:139-352):
//   Q_lm = sum_i w_i G_m(theta_i) ytilde_l^m(theta_i)
//
// Layouts: coefficients q[field][lm] (float2, m-major lm order); the Fourier
// intermediate fm[field][m][ilat] (float2, latitude contiguous).
#pragma once
#include "ts_common.cuh"

// ---------------------------------------------------------------- synthesis
//
// One thread per northern latitude, F fields per thread (the recurrence is
// shared by the F fields).  grid = (ceil(nh / blockDim), mmax+1, ceil(nf / F)).
// y0 always carries even (l-m) and y1 odd (l-m), so
//   F(north) = E + O,  F(south) = E - O   (ytilde_l^m(-x) = (-1)^(l-m) ytilde).
// Dynamic shared memory: (K + K*F) float2, K = lmax - m + 1 <= lmax + 1.
template <int F>
__global__ void __launch_bounds__(128)
ts_leg_synth_f32(TsLegTab t, TsFields q, float2 *__restrict__ fm, long fm_stride, int nfields) {
  extern __shared__ float2 ts_smem_ls[];
  const int m = blockIdx.y;
  const int f0 = blockIdx.z * F;
  const int K = t.lmax - m + 1;
  const long base = ts_lm_base(t.lmax, m);
  float2 *sab = ts_smem_ls;
  float2 *sq = ts_smem_ls + K;
  for (int i = threadIdx.x; i < K; i += blockDim.x) sab[i] = t.ab[base + i];
#pragma unroll
  for (int f = 0; f < F; f++) {
    const bool ok = f0 + f < nfields;
    const float2 *src = ok ? ts_field(q, f0 + f) + base : nullptr;
    for (int i = threadIdx.x; i < K; i += blockDim.x)
      sq[i * F + f] = ok ? src[i] : make_float2(0.f, 0.f);
  }
  __syncthreads();

  const int lat = blockIdx.x * blockDim.x + threadIdx.x;
  if (lat >= t.nh) return;
  const float ct = t.ct[lat];
  const float st = t.st[lat];
  float y0;
  int ny;
  ts_sinpow(st, m, y0, ny);
  y0 *= t.amm[m];
  float y1 = (m < t.lmax) ? sab[1].x * ct * y0 : 0.0f;

  float2 aE[F], aO[F];
#pragma unroll
  for (int f = 0; f < F; f++) {
    aE[f] = make_float2(0.f, 0.f);
    aO[f] = make_float2(0.f, 0.f);
  }
  int i = 0;  // l - m
  while (true) {
    if (ny == 0) {
#pragma unroll
      for (int f = 0; f < F; f++) {
        const float2 qa = sq[i * F + f];
        aE[f].x = fmaf(y0, qa.x, aE[f].x);
        aE[f].y = fmaf(y0, qa.y, aE[f].y);
      }
      if (i + 1 < K) {
#pragma unroll
        for (int f = 0; f < F; f++) {
          const float2 qb = sq[(i + 1) * F + f];
          aO[f].x = fmaf(y1, qb.x, aO[f].x);
          aO[f].y = fmaf(y1, qb.y, aO[f].y);
        }
      }
    } else if (fabsf(y0) > TS_RESCALE_THR) {
      ny += 1;
      y0 *= TS_INV_SCALE;
      y1 *= TS_INV_SCALE;
    }
    if (i + 2 >= K) break;
    const float2 a0 = sab[i + 2];
    const float2 a1 = (i + 3 < K) ? sab[i + 3] : make_float2(0.f, 0.f);
    const float t0 = a0.x * ct * y1 + a0.y * y0;
    y1 = a1.x * ct * t0 + a1.y * y1;
    y0 = t0;
    i += 2;
  }
  const int south = t.nlat - 1 - lat;
#pragma unroll
  for (int f = 0; f < F; f++) {
    if (f0 + f >= nfields) break;
    float2 *dst = fm + (long)(f0 + f) * fm_stride + (long)m * t.nlat;
    dst[lat] = c_add(aE[f], aO[f]);
    if (south != lat) dst[south] = c_sub(aE[f], aO[f]);
  }
}

// ----------------------------------------------------------------- analysis
//
// One CTA per (m, group of F fields); threads own K northern latitudes each
// (lat = tid + k*blockDim).  Each thread keeps its folded weighted inputs
//   wp = (G_north + G_south) * w,  wm = (G_north - G_south) * w
// in registers, accumulates P l-pairs of partial sums, then the CTA reduces:
// a butterfly reduce-scatter inside each warp followed by a sum over warps in
// shared memory.  The reduced values go through the epilogue functor `Epi`,
// which receives, for one (lm, re|im) component, the F values of the group.

// Butterfly reduce-scatter of N values over the 32 lanes of a warp.  On
// return lane holds `cnt` reduced values at original indices base..base+cnt-1;
// when N < 32 several lanes hold the same values and only lanes with
// (lane & dup_mask) == 0 should write them.
template <int N>
TS_DEV void ts_warp_reduce_scatter(float (&v)[N], int lane, int &base) {
  int n = N;
  base = 0;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    if (n > 1) {
      const int h = n >> 1;
      const bool upper = (lane & o) != 0;
#pragma unroll
      for (int i = 0; i < N / 2; i++) {
        if (i < h) {
          const float send = upper ? v[i] : v[h + i];
          const float keep = upper ? v[h + i] : v[i];
          v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
      if (upper) base += h;
      n = h;
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    }
  }
}

// Store epilogue: out[field][lm] component c.
struct TsAnalysStore {
  float2 *out;
  long out_stride;
  TS_DEV void operator()(long lm, int comp, const float *vals, int f0, int nf, int F) const {
    for (int f = 0; f < nf; f++) {
      float *dst = reinterpret_cast<float *>(out + (long)(f0 + f) * out_stride + lm);
      dst[comp] = vals[f];
    }
  }
};

// per_cta <= F fields per CTA (a model groups whole instances per CTA).
// lchunk > 0 splits each m's degrees over CTAs (blockIdx.z: degrees
// i = l - m in [z*lchunk, (z+1)*lchunk), lchunk a multiple of 2P): a CTA
// advances the recurrence without reducing up to its chunk, so small grids
// still fill the GPU; 0 = one CTA per m.
template <int F, int K, int P, class Epi>
__global__ void __launch_bounds__(256)
ts_leg_analys_f32(TsLegTab t, const float2 *__restrict__ g, long g_stride, Epi epi,
                  int nfields, int per_cta, int lchunk) {
  constexpr int N = 4 * P * F;  // (p, comp4, f) values per span
  constexpr int CNT = N >= 32 ? N / 32 : 1;
  extern __shared__ float ts_smem_la[];
  const int m = blockIdx.x;
  const int f0 = blockIdx.y * per_cta;
  const int nf = min(per_cta, nfields - f0);
  const int Km = t.lmax - m + 1;
  const int c_begin = lchunk ? (int)blockIdx.z * lchunk : 0;
  const int c_end = lchunk ? min(Km, c_begin + lchunk) : Km;
  if (c_begin >= Km) return;
  const long base = ts_lm_base(t.lmax, m);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int W = blockDim.x >> 5;

  float2 *sab = reinterpret_cast<float2 *>(ts_smem_la);   // [Km]
  float *red = ts_smem_la + 2 * (t.lmax + 1);              // [W][N]
  float *res = red + W * N;                                 // [N]
  for (int i = tid; i < Km; i += blockDim.x) sab[i] = t.ab[base + i];

  float ctv[K], y0v[K], y1v[K];
  int nyv[K];
  float2 wp[K][F], wm[K][F];
  const float amm = t.amm[m];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int lat = tid + k * blockDim.x;
    float ct = 0.f, st = 0.f, w = 0.f;
    const bool ok = lat < t.nh;
    if (ok) {
      ct = t.ct[lat];
      st = t.st[lat];
      w = t.wq[lat];
    }
    const int south = t.nlat - 1 - lat;
#pragma unroll
    for (int f = 0; f < F; f++) {
      float2 gn = make_float2(0.f, 0.f), gs = make_float2(0.f, 0.f);
      if (ok && f < nf) {
        const float2 *src = g + (long)(f0 + f) * g_stride + (long)m * t.nlat;
        gn = src[lat];
        gs = (south != lat) ? src[south] : make_float2(0.f, 0.f);
      }
      wp[k][f] = c_scale(c_add(gn, gs), w);
      wm[k][f] = c_scale(c_sub(gn, gs), w);
    }
    ctv[k] = ct;
    float y;
    int ny;
    ts_sinpow(st, m, y, ny);
    y0v[k] = ok ? y * amm : 0.0f;
    nyv[k] = ok ? ny : 1;  // out-of-range lanes never contribute
    y1v[k] = (m < t.lmax) ? sab[1].x * ct * y0v[k] : 0.0f;
  }

  for (int i0 = 0; i0 < c_begin; i0 += 2 * P) {  // recurrence only, up to the chunk
#pragma unroll
    for (int p = 0; p < P; p++) {
      const int i = i0 + 2 * p;
#pragma unroll
      for (int k = 0; k < K; k++)
        if (nyv[k] != 0 && fabsf(y0v[k]) > TS_RESCALE_THR) {
          nyv[k] += 1;
          y0v[k] *= TS_INV_SCALE;
          y1v[k] *= TS_INV_SCALE;
        }
      if (i + 2 < Km) {
        const float2 a0 = sab[i + 2];
        const float2 a1 = (i + 3 < Km) ? sab[i + 3] : make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < K; k++) {
          const float t0 = a0.x * ctv[k] * y1v[k] + a0.y * y0v[k];
          y1v[k] = a1.x * ctv[k] * t0 + a1.y * y1v[k];
          y0v[k] = t0;
        }
      }
    }
  }
  for (int i0 = c_begin; i0 < c_end; i0 += 2 * P) {
    float v[N];
#pragma unroll
    for (int j = 0; j < N; j++) v[j] = 0.f;
#pragma unroll
    for (int p = 0; p < P; p++) {
      const int i = i0 + 2 * p;
      if (i < Km) {
#pragma unroll
        for (int k = 0; k < K; k++) {
          if (nyv[k] == 0) {
#pragma unroll
            for (int f = 0; f < F; f++) {
              v[(p * 4 + 0) * F + f] = fmaf(wp[k][f].x, y0v[k], v[(p * 4 + 0) * F + f]);
              v[(p * 4 + 1) * F + f] = fmaf(wp[k][f].y, y0v[k], v[(p * 4 + 1) * F + f]);
              v[(p * 4 + 2) * F + f] = fmaf(wm[k][f].x, y1v[k], v[(p * 4 + 2) * F + f]);
              v[(p * 4 + 3) * F + f] = fmaf(wm[k][f].y, y1v[k], v[(p * 4 + 3) * F + f]);
            }
          } else if (fabsf(y0v[k]) > TS_RESCALE_THR) {
            nyv[k] += 1;
            y0v[k] *= TS_INV_SCALE;
            y1v[k] *= TS_INV_SCALE;
          }
        }
        if (i + 2 < Km) {
          const float2 a0 = sab[i + 2];
          const float2 a1 = (i + 3 < Km) ? sab[i + 3] : make_float2(0.f, 0.f);
#pragma unroll
          for (int k = 0; k < K; k++) {
            const float t0 = a0.x * ctv[k] * y1v[k] + a0.y * y0v[k];
            y1v[k] = a1.x * ctv[k] * t0 + a1.y * y1v[k];
            y0v[k] = t0;
          }
        }
      }
    }
    int rbase;
    ts_warp_reduce_scatter<N>(v, lane, rbase);
    const bool writer = (N >= 32) || ((lane & ((32 / (N < 32 ? N : 32)) - 1)) == 0);
    if (writer) {
#pragma unroll
      for (int j = 0; j < CNT; j++) red[warp * N + rbase + j] = v[j];
    }
    __syncthreads();
    for (int j = tid; j < N; j += blockDim.x) {
      float s = 0.f;
      for (int w = 0; w < W; w++) s += red[w * N + j];
      res[j] = s;
    }
    __syncthreads();
    // 2P l-values x 2 components per span
    for (int j = tid; j < 4 * P; j += blockDim.x) {
      const int p = j >> 2, c = j & 3;
      const int i = i0 + 2 * p + (c >> 1);
      if (i < c_end) epi(base + i, c & 1, res + (p * 4 + c) * F, f0, nf, F);
    }
    __syncthreads();
  }
}
