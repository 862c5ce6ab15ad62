// Longitude stage on a two-phase shared-memory FFT.
//
// The real-row conventions are those of fourier.cuh: a row of nphi real
// values is a half-length complex row z[n] = x[2n] + i x[2n+1] of H = nphi/2
// points, and
//   synthesis: Z[k] = (X[k] + conj X[H-k]) + i e^{+2 pi i k/nphi} (X[k] - conj X[H-k]),
//              z = FFT_H^{+}(Z);
//   analysis:  Z = FFT_H^{-}(z),
//              X[k] = (Z[k] + conj Z[H-k])/2 - i e^{-2 pi i k/nphi} (Z[k] - conj Z[H-k])/2.
//
// A CTA holds R rows in shared memory and transforms them in place, with
// H = P * Q split as (w = e^{2 pi i/H})
//   k = k1 + P k2,  n = Q n1 + n2   (k1, n1 < P;  k2, n2 < Q)
//   z[Q n1 + n2] = sum_k1 e^{2 pi i n1 k1/P} w^{n2 k1} sum_k2 Z[k1 + P k2] e^{2 pi i n2 k2/Q}.
// Phase 1 gives every thread one (row, k1) and a Q-point DFT in registers;
// phase 2 one (row, n2) and a P-point DFT.  The analysis runs the mirror
// image (P-point DFTs, conjugate twiddles, Q-point DFTs).  Between the
// phases a row is stored transposed, element (k1, n2) at n2 (P+1) + k1; with
// P even the odd pitch P+1, and an odd row pitch, make every phase's shared
// accesses conflict-free (lanes step through consecutive k1, n2 or rows).
// The DFTs inside a thread are Stockham sequences over compile-time radices
// (4, 2, 3) whose twiddles are compile-time constants.
//
// Global traffic: spectra are read and written as fm[m][lat] with
// consecutive threads on consecutive latitudes; grid rows as whole rows.
#pragma once
#include "ts_common.cuh"

// ------------------------------------------------- compile-time helpers
template <int V>
struct TsIC {
  static constexpr int value = V;
};

// f(TsIC<B>{}), f(TsIC<B+1>{}), ..., f(TsIC<E-1>{})
template <int B, int E, class F>
TS_DEV void ts_sfor(F &&f) {
  if constexpr (B < E) {
    f(TsIC<B>{});
    ts_sfor<B + 1, E>(f);
  }
}

// cos and sin of 2 pi num/den, evaluated by the compiler: the angle is
// reduced to [-pi, pi] exactly (integer arithmetic) and summed as a Taylor
// series in double precision (16 terms: remainder below 1e-18 at |x| = pi).
constexpr double ts_cx_pi = 3.14159265358979323846264338327950288;
__host__ __device__ constexpr double ts_cx_angle(long num, long den) {
  long n = num % den;
  if (n < 0) n += den;
  if (2 * n > den) n -= den;
  return 2.0 * ts_cx_pi * (double)n / (double)den;
}
__host__ __device__ constexpr double ts_cx_sin_series(double x) {
  double t = x, s = x;
  for (int i = 1; i < 16; i++) {
    t *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    s += t;
  }
  return s;
}
__host__ __device__ constexpr double ts_cx_cos_series(double x) {
  double t = 1.0, s = 1.0;
  for (int i = 1; i < 16; i++) {
    t *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    s += t;
  }
  return s;
}
__host__ __device__ constexpr float ts_cx_cos(long num, long den) { return (float)ts_cx_cos_series(ts_cx_angle(num, den)); }
__host__ __device__ constexpr float ts_cx_sin(long num, long den) { return (float)ts_cx_sin_series(ts_cx_angle(num, den)); }

// a * e^{SIGN 2 pi i NUM/DEN}; quarter turns are exact swaps and negations
template <long NUM, long DEN, int SIGN>
TS_DEV float2 ts_twc(float2 a) {
  constexpr long n = ((NUM % DEN) + DEN) % DEN;
  if constexpr (n == 0) {
    return a;
  } else if constexpr (2 * n == DEN) {
    return make_float2(-a.x, -a.y);
  } else if constexpr (4 * n == DEN) {
    return SIGN > 0 ? c_mul_i(a) : c_mul_negi(a);
  } else if constexpr (4 * n == 3 * DEN) {
    return SIGN > 0 ? c_mul_negi(a) : c_mul_i(a);
  } else {
    constexpr float c = ts_cx_cos(n, DEN);
    constexpr float s = SIGN * ts_cx_sin(n, DEN);
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

template <int M>
struct TsRadix {
  static constexpr int value = (M % 4 == 0) ? 4 : (M % 2 == 0) ? 2 : 3;
};

// R-point DFT (R = 2, 3, 4) of a[0..R), sign SIGN
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
    const float h = SIGN * 0.8660254037844386f;  // sin(2 pi/3)
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

// Stockham stage NS of an N-point DFT in registers, then the remaining ones
template <int N, int NS, int SIGN>
TS_DEV void ts_dft_rec(float2 (&x)[N]) {
  if constexpr (NS < N) {
    constexpr int R = TsRadix<N / NS>::value;
    constexpr int MR = N / R;
    float2 y[N];
    ts_sfor<0, MR>([&](auto tc) {
      constexpr int t = decltype(tc)::value;
      constexpr int j = t % NS;
      float2 a[R];
      ts_sfor<0, R>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        a[q] = ts_twc<(long)q * j, (long)NS * R, SIGN>(x[t + q * MR]);
      });
      ts_butterfly<R, SIGN>(a);
      ts_sfor<0, R>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        y[(t - j) * R + j + q * NS] = a[q];
      });
    });
#pragma unroll
    for (int i = 0; i < N; i++) x[i] = y[i];
    ts_dft_rec<N, NS * R, SIGN>(x);
  }
}

// N-point DFT, natural order in and out: x[k] <- sum_n x[n] e^{SIGN 2 pi i nk/N}
template <int N, int SIGN>
TS_DEV void ts_dft(float2 (&x)[N]) {
  ts_dft_rec<N, 1, SIGN>(x);
}

// ------------------------------------------------------------- geometry
template <int P_, int Q_, int R_>
struct TsF2 {
  static constexpr int P = P_, Q = Q_, R = R_, H = P_ * Q_, T = P_ * R_;
  static constexpr int P1 = P_ + 1;        // pitch of the transposed view
  static constexpr int RP = (H + Q_) | 1;  // row pitch: odd, >= Q (P+1) = H + Q
  static constexpr int TWQ = Q_ * P1;      // inter-phase twiddles [n2][k1]
};

// Thread -> (row r, k1) of the phases that run one Q-point DFT per (r, k1).
// With R >= 16 rows a half-warp takes one k1 of 16 consecutive rows: the odd
// row pitch spreads them over 16 distinct banks and they share one twiddle
// (rows first would put two rows in some half-warps, whose columns k1 and
// k1 + 16 collide); with fewer rows the rows stay together.
template <class C>
TS_DEV void ts_f2_rk(int tid, int &r, int &k1) {
  if constexpr (C::R >= 16) {
    k1 = tid / C::R;
    r = tid - k1 * C::R;
  } else {
    r = tid / C::P;
    k1 = tid - r * C::P;
  }
}

// twq[n2 (P+1) + k1] = w^{n2 k1} = tw[2 n2 k1] (2 n2 k1 <= 2 (P-1)(Q-1) < nphi)
template <class C>
TS_DEV void ts_f2_twq(float2 *twq, const TsFftTab &ft) {
  for (int i = threadIdx.x; i < C::Q * C::P; i += C::T) {
    const int n2 = i / C::P, k1 = i - n2 * C::P;
    twq[n2 * C::P1 + k1] = __ldg(ft.tw + 2 * n2 * k1);
  }
}

// z = FFT_H^{+}(Z) of the R rows at b (natural order in and out)
template <class C>
TS_DEV void ts_f2_inverse(float2 *b, const float2 *twq) {
  const int tid = threadIdx.x;
  {
    int r, k1;
  ts_f2_rk<C>(tid, r, k1);
    float2 *row = b + r * C::RP;
    float2 x[C::Q];
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) x[k2] = row[k1 + C::P * k2];
    ts_dft<C::Q, +1>(x);
#pragma unroll
    for (int n2 = 1; n2 < C::Q; n2++) x[n2] = c_mul(x[n2], twq[n2 * C::P1 + k1]);
    __syncthreads();
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) row[n2 * C::P1 + k1] = x[n2];
    __syncthreads();
  }
  {
    const bool act = tid < C::Q * C::R;
    const int r = tid / C::Q, n2 = tid - r * C::Q;
    float2 *row = b + r * C::RP;
    float2 x[C::P];
    if (act) {
#pragma unroll
      for (int k1 = 0; k1 < C::P; k1++) x[k1] = row[n2 * C::P1 + k1];
      ts_dft<C::P, +1>(x);
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int n1 = 0; n1 < C::P; n1++) row[C::Q * n1 + n2] = x[n1];
    }
    __syncthreads();
  }
}

// Z = FFT_H^{-}(z) of the R rows at b (natural order in and out)
template <class C>
TS_DEV void ts_f2_forward(float2 *b, const float2 *twq) {
  const int tid = threadIdx.x;
  {
    const bool act = tid < C::Q * C::R;
    const int r = tid / C::Q, n2 = tid - r * C::Q;
    float2 *row = b + r * C::RP;
    float2 x[C::P];
    if (act) {
#pragma unroll
      for (int n1 = 0; n1 < C::P; n1++) x[n1] = row[C::Q * n1 + n2];
      ts_dft<C::P, -1>(x);
#pragma unroll
      for (int k1 = 1; k1 < C::P; k1++) x[k1] = c_mul(x[k1], c_conj(twq[n2 * C::P1 + k1]));
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int k1 = 0; k1 < C::P; k1++) row[n2 * C::P1 + k1] = x[k1];
    }
    __syncthreads();
  }
  {
    int r, k1;
  ts_f2_rk<C>(tid, r, k1);
    float2 *row = b + r * C::RP;
    float2 x[C::Q];
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) x[n2] = row[n2 * C::P1 + k1];
    ts_dft<C::Q, -1>(x);
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) row[k1 + C::P * k2] = x[k2];
    __syncthreads();
  }
}

// ts_f2_inverse whose second phase writes z straight to the grid rows
// (16 consecutive n2 per half-warp: 128-byte runs), skipping the staging of
// the result in shared memory
template <class C, class LatOf>
TS_DEV void ts_f2_inverse_out(float2 *b, const float2 *twq, float *__restrict__ dst, int nphi,
                              LatOf lat_of) {
  const int tid = threadIdx.x;
  {
    int r, k1;
  ts_f2_rk<C>(tid, r, k1);
    float2 *row = b + r * C::RP;
    float2 x[C::Q];
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) x[k2] = row[k1 + C::P * k2];
    ts_dft<C::Q, +1>(x);
#pragma unroll
    for (int n2 = 1; n2 < C::Q; n2++) x[n2] = c_mul(x[n2], twq[n2 * C::P1 + k1]);
    __syncthreads();
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) row[n2 * C::P1 + k1] = x[n2];
    __syncthreads();
  }
  if (tid < C::Q * C::R) {
    const int r = tid / C::Q, n2 = tid - r * C::Q;
    const int lat = lat_of(r);
    const float2 *row = b + r * C::RP;
    float2 x[C::P];
#pragma unroll
    for (int k1 = 0; k1 < C::P; k1++) x[k1] = row[n2 * C::P1 + k1];
    ts_dft<C::P, +1>(x);
    if (lat >= 0) {
      float2 *out = reinterpret_cast<float2 *>(dst + (long)lat * nphi) + n2;
#pragma unroll
      for (int n1 = 0; n1 < C::P; n1++) out[C::Q * n1] = x[n1];
    }
  }
}

// grid rows leave shared memory by bulk copies (one per row, issued by one
// thread; the async proxy reads the staging, so the writes are fenced first)
TS_DEV void ts_f2_fence_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
TS_DEV void ts_f2_bulk_s2g(void *dst, const void *src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(
                   reinterpret_cast<unsigned long long>(dst)),
               "r"((unsigned)__cvta_generic_to_shared(src)), "r"(bytes)
               : "memory");
}
TS_DEV void ts_f2_bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
TS_DEV void ts_f2_bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// ts_f2_inverse whose second phase stages z in natural order (row pitch H,
// 16-byte aligned rows) and writes each grid row with one bulk copy.  Needs
// dst 16-byte aligned and nphi a multiple of 4 (the caller checks).
template <class C, class LatOf>
TS_DEV void ts_f2_inverse_bulk(float2 *b, const float2 *twq, float *__restrict__ dst, int nphi,
                               LatOf lat_of) {
  const int tid = threadIdx.x;
  {
    int r, k1;
    ts_f2_rk<C>(tid, r, k1);
    float2 *row = b + r * C::RP;
    float2 x[C::Q];
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) x[k2] = row[k1 + C::P * k2];
    ts_dft<C::Q, +1>(x);
#pragma unroll
    for (int n2 = 1; n2 < C::Q; n2++) x[n2] = c_mul(x[n2], twq[n2 * C::P1 + k1]);
    __syncthreads();
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) row[n2 * C::P1 + k1] = x[n2];
    __syncthreads();
  }
  const bool act = tid < C::Q * C::R;
  const int r = tid / C::Q, n2 = tid - r * C::Q;
  float2 x[C::P];
  if (act) {
    const float2 *row = b + r * C::RP;
#pragma unroll
    for (int k1 = 0; k1 < C::P; k1++) x[k1] = row[n2 * C::P1 + k1];
    ts_dft<C::P, +1>(x);
  }
  __syncthreads();
  if (act) {
    float2 *srow = b + r * C::H;
#pragma unroll
    for (int n1 = 0; n1 < C::P; n1++) srow[C::Q * n1 + n2] = x[n1];
    ts_f2_fence_async();
  }
  __syncthreads();
  if (tid < C::R) {
    const int lat = lat_of(tid);
    if (lat >= 0) {
      ts_f2_bulk_s2g(dst + (long)lat * nphi, b + tid * C::H, (unsigned)(nphi * sizeof(float)));
      ts_f2_bulk_commit();
      ts_f2_bulk_wait_read();
    }
  }
}

// ts_f2_forward whose first phase reads z straight from the grid rows
template <class C, class LatOf>
TS_DEV void ts_f2_forward_in(float2 *b, const float2 *twq, const float *__restrict__ src, int nphi,
                             LatOf lat_of) {
  const int tid = threadIdx.x;
  if (tid < C::Q * C::R) {
    const int r = tid / C::Q, n2 = tid - r * C::Q;
    const int lat = lat_of(r);
    float2 x[C::P];
    if (lat >= 0) {
      const float2 *in = reinterpret_cast<const float2 *>(src + (long)lat * nphi) + n2;
#pragma unroll
      for (int n1 = 0; n1 < C::P; n1++) x[n1] = in[C::Q * n1];
    } else {
#pragma unroll
      for (int n1 = 0; n1 < C::P; n1++) x[n1] = make_float2(0.f, 0.f);
    }
    ts_dft<C::P, -1>(x);
#pragma unroll
    for (int k1 = 1; k1 < C::P; k1++) x[k1] = c_mul(x[k1], c_conj(twq[n2 * C::P1 + k1]));
    float2 *row = b + r * C::RP;
#pragma unroll
    for (int k1 = 0; k1 < C::P; k1++) row[n2 * C::P1 + k1] = x[k1];
  }
  __syncthreads();
  {
    int r, k1;
  ts_f2_rk<C>(tid, r, k1);
    float2 *row = b + r * C::RP;
    float2 x[C::Q];
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) x[n2] = row[n2 * C::P1 + k1];
    ts_dft<C::Q, -1>(x);
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) row[k1 + C::P * k2] = x[k2];
    __syncthreads();
  }
}

// Z of the synthesis for the CTA's rows from the spectra src[k*nlat + lat]
// of one field.  lat_of(r) < 0 marks a row without a latitude (zeros).
// Item i is the pair (k, H-k), k = i / R, of row i % R: consecutive threads
// read consecutive latitudes.  Every load of a thread is issued before the
// first is used.  One twiddle serves both members of a pair: with
// s = X[k] + conj X[H-k] and u = i e^{2 pi i k/nphi} (X[k] - conj X[H-k]),
// Z[k] = s + u and, as e^{2 pi i (H-k)/nphi} = -conj e^{2 pi i k/nphi},
// Z[H-k] = conj(s - u).
// NS fields at once: field s from src + s * src_stride into the row block at
// b + s * bs (the loads of every field are in flight together).
template <class C, int NS, class LatOf>
TS_DEV void ts_f2_pack_n(float2 *b, long bs, const float2 *__restrict__ src, long src_stride,
                         const TsFftTab &ft, LatOf lat_of) {
  // thread t keeps row t % R and takes the pairs k = t / R + P j (T = P R)
  constexpr int H = C::H, NK = H / 2 + 1, NI = (NK + C::P - 1) / C::P;
  const int r = threadIdx.x % C::R, k0 = threadIdx.x / C::R;
  const int lat = lat_of(r);
  float2 xk[NS][NI], xh[NS][NI];
#pragma unroll
  for (int s = 0; s < NS; s++) {
    const float2 *col = src + s * src_stride + (lat >= 0 ? lat : 0);
#pragma unroll
    for (int j = 0; j < NI; j++) {
      const int kk = k0 + C::P * j;
      xk[s][j] = make_float2(0.f, 0.f);
      xh[s][j] = make_float2(0.f, 0.f);
      if (lat >= 0 && kk < NK) {
        if (kk <= ft.mmax) xk[s][j] = col[(long)kk * ft.nlat];
        if (H - kk <= ft.mmax) xh[s][j] = col[(long)(H - kk) * ft.nlat];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NI; j++) {
    const int kk = k0 + C::P * j;
    if (kk < NK) {
      const int h = H - kk;
      const float2 t = __ldg(ft.tw + kk);
#pragma unroll
      for (int s = 0; s < NS; s++) {
        float2 *row = b + s * bs + r * C::RP;
        const float2 x = kk == 0 ? make_float2(xk[s][j].x, 0.f) : xk[s][j];
        const float2 ch = c_conj(xh[s][j]);
        const float2 sp = c_add(x, ch);
        const float2 u = c_mul_i(c_mul(c_sub(x, ch), t));
        row[kk] = c_add(sp, u);
        if (kk > 0 && kk < h) row[h] = c_conj(c_sub(sp, u));
      }
    }
  }
}

template <class C, class LatOf>
TS_DEV void ts_f2_pack(float2 *b, const float2 *__restrict__ src, const TsFftTab &ft,
                       LatOf lat_of) {
  ts_f2_pack_n<C, 1>(b, 0, src, 0, ft, lat_of);
}

// 2 X[k] of the analysis from the forward-transformed row and the twiddle
// t = e^{2 pi i k/nphi}: with a = Z[k], b = conj Z[H-k],
// 2 X[k] = (a + b) - i conj(t) (a - b)
template <class C>
TS_DEV float2 ts_f2_xk2(const float2 *row, int k, float2 t) {
  const float2 zk = row[k];
  const float2 zh = c_conj(row[k == 0 ? 0 : C::H - k]);
  const float2 sm = c_add(zk, zh), d = c_sub(zk, zh);
  // -i conj(t) d = (d.y t.x - d.x t.y, -(d.x t.x + d.y t.y))
  return make_float2(sm.x + (d.y * t.x - d.x * t.y), sm.y - (d.x * t.x + d.y * t.y));
}

// X[k] of the analysis from the forward-transformed row
template <class C>
TS_DEV float2 ts_f2_xk(const float2 *row, int k, const TsFftTab &ft) {
  return c_scale(ts_f2_xk2<C>(row, k, __ldg(ft.tw + k)), 0.5f);
}

// X[k], k <= mmax, of the CTA's rows -> dst[k*nlat + lat]
template <class C, class LatOf>
TS_DEV void ts_f2_unpack(const float2 *b, float2 *__restrict__ dst, const TsFftTab &ft,
                         LatOf lat_of) {
  // thread t keeps row t % R and takes k = t / R + P j
  const int r = threadIdx.x % C::R;
  const int lat = lat_of(r);
  if (lat < 0) return;
  const float2 *row = b + r * C::RP;
  float2 *col = dst + lat;
  for (int k = threadIdx.x / C::R; k <= ft.mmax; k += C::P)
    col[(long)k * ft.nlat] = ts_f2_xk<C>(row, k, ft);
}

// grid rows: b <-> rows of src/dst (row `lat` starts at lat*nphi floats).
// Element i = (row i / H, column i % H), i = t + T j: when T is a multiple
// of H a thread keeps one column and steps through rows.
template <class C, class F>
TS_DEV void ts_f2_for_rows(F &&f) {
  constexpr int NI = (C::R * C::H + C::T - 1) / C::T;
  if constexpr (C::T % C::H == 0) {
    const int n = threadIdx.x % C::H, r0 = threadIdx.x / C::H;
#pragma unroll
    for (int j = 0; j < NI; j++) f(j, r0 + (C::T / C::H) * j, n);
  } else {
#pragma unroll
    for (int j = 0; j < NI; j++) {
      const int i = threadIdx.x + j * C::T;
      if (i < C::R * C::H) f(j, i / C::H, i % C::H);
    }
  }
}

template <class C, class LatOf>
TS_DEV void ts_f2_load_rows(float2 *b, const float *__restrict__ src, int nphi, LatOf lat_of) {
  constexpr int NI = (C::R * C::H + C::T - 1) / C::T;
  float2 v[NI];
  ts_f2_for_rows<C>([&](int j, int r, int n) {
    const int lat = lat_of(r);
    v[j] = lat >= 0 ? reinterpret_cast<const float2 *>(src + (long)lat * nphi)[n]
                    : make_float2(0.f, 0.f);
  });
  ts_f2_for_rows<C>([&](int j, int r, int n) { b[r * C::RP + n] = v[j]; });
}

template <class C, class LatOf>
TS_DEV void ts_f2_store_rows(const float2 *b, float *__restrict__ dst, int nphi, LatOf lat_of) {
  ts_f2_for_rows<C>([&](int, int r, int n) {
    const int lat = lat_of(r);
    if (lat >= 0) reinterpret_cast<float2 *>(dst + (long)lat * nphi)[n] = b[r * C::RP + n];
  });
}

// ------------------------------------------------- W image of the TC path
//
// Tensor-core plans consume the analysis as W_par = w (G_north +- G_south)
// in the MMA's byte image (TsTcImg.w).  A paired CTA holds R/2 northern
// latitudes lat0 + j in rows j and their southern mirrors in rows R/2 + j
// (a row without a latitude, or the equator's repeat, reads as zero), and
// writes the folded, weighted values: with R/2 = 8 and lat0 a multiple of 8,
// every (m, parity, re|im) run covers one whole 32-byte sector of the image.
// w_kmin (null: none) holds, per 32-latitude chunk and parity, the order m
// from which the polar-skipped analysis never reads that chunk: writes of
// those (m, parity) blocks are left out.
template <class C>
TS_DEV void ts_f2_write_w(const float2 *b, int lat0, long f, const TsFftTab &ft,
                          const float *__restrict__ wq, char *wimg, int nfb, int fpb, int nlc,
                          int nh, const int *__restrict__ w_kmin) {
  constexpr int NPR = C::R / 2;
  const long fb = f / fpb;
  const int fl = (int)(f - fb * fpb);
  // thread t keeps latitude pair t % NPR and takes m = t / NPR + 2P j
  const int j = threadIdx.x % NPR;
  const int lat = lat0 + j;
  if (lat >= nh) return;
  const float2 *rn = b + j * C::RP, *rs = b + (NPR + j) * C::RP;
  const bool south = ft.nlat - 1 - lat != lat;
  const float w = 0.5f * __ldg(wq + lat);  // times 2 X[k] of both rows
  // byte offsets of (row 2 fl + re|im, column lat % 32) inside a 16 KB block,
  // and of this field block's chunk: block (((k nfb + fb) 2 + par) nlc + lat / 32)
  const int o_re = ts_swz_img(2 * fl, lat & 31), o_im = ts_swz_img(2 * fl + 1, lat & 31);
  char *base = wimg + ((long)fb * 2 * nlc + (lat >> 5)) * 16384;
  const long kstep = (long)nfb * 2 * nlc * 16384, pstep = (long)nlc * 16384;
  // k groups g = threadIdx.x / NPR (2P of them), permuted so that the two
  // halves of a half-warp take k 8 apart: their row reads then fall in
  // disjoint banks (a bijection when 2P is a multiple of 16)
  const int g = threadIdx.x / NPR;
  const int k0 = (2 * C::P) % 16 == 0 ? (g & ~15) + ((g & 1) << 3) + ((g >> 1) & 7) : g;
  const int kl0 = w_kmin ? __ldg(w_kmin + 2 * (lat >> 5)) : ft.mmax + 1;
  const int kl1 = w_kmin ? __ldg(w_kmin + 2 * (lat >> 5) + 1) : ft.mmax + 1;
  const int kend = min(ft.mmax + 1, max(kl0, kl1));
  for (int k = k0; k < kend; k += 2 * C::P) {
    const bool e0 = k < kl0, e1 = k < kl1;
    const float2 t = __ldg(ft.tw + k);
    const float2 xn = ts_f2_xk2<C>(rn, k, t);
    const float2 xs = south ? ts_f2_xk2<C>(rs, k, t) : make_float2(0.f, 0.f);
    char *blk = base + k * kstep;
    if (e0) {
      *reinterpret_cast<float *>(blk + o_re) = w * (xn.x + xs.x);
      *reinterpret_cast<float *>(blk + o_im) = w * (xn.y + xs.y);
    }
    if (e1) {
      *reinterpret_cast<float *>(blk + pstep + o_re) = w * (xn.x - xs.x);
      *reinterpret_cast<float *>(blk + pstep + o_im) = w * (xn.y - xs.y);
    }
  }
}

// latitude of row r: plain CTAs hold lat0 + r; paired CTAs northern rows
// lat0 + r (r < R/2) and their mirrors
template <class C, bool PAIRED>
struct TsF2Rows {
  int lat0, nlat, nh;
  TS_DEV int operator()(int r) const {
    if constexpr (PAIRED) {
      const int j = r < C::R / 2 ? r : r - C::R / 2;
      const int latN = lat0 + j;
      if (latN >= nh) return -1;
      if (r < C::R / 2) return latN;
      const int latS = nlat - 1 - latN;
      return latS != latN ? latS : -1;
    } else {
      const int lat = lat0 + r;
      return lat < nlat ? lat : -1;
    }
  }
};

// Shared memory of a CTA with NB row blocks (floats2):
//   twq[TWQ] | NB x rows[R][RP]
template <class C>
constexpr long ts_f2_smem_bytes(int nb) {
  return (long)sizeof(float2) * (C::TWQ + (long)nb * C::R * C::RP);
}

// ---------------------------------------------------------------- kernels

// Resident CTAs per SM asked of the register allocator.  Transform kernels
// with P <= 24: 1152 threads per SM (<= 56 registers each), else whatever
// fits.  The fused phase keeps every species' P grid points of a row in
// registers (~170 registers): no limit.
#define TS_F2_MINB(P, R) ((P) <= 24 ? 1152 / ((P) * (R)) : 1)
#define TS_F2_PHASE_MINB(P, R) 1

// fm[field][m][lat] -> spat[field][lat][phi].  grid = (ceil(nlat/R), fields),
// block = P*R.  Rows leave by bulk copies when the field's grid is 16-byte
// aligned (fewer, larger memory instructions), else by per-thread stores.
template <int P, int Q, int R>
__global__ void __launch_bounds__(P *R, TS_F2_MINB(P, R))
ts_f2_synth(TsFftTab ft, const float2 *__restrict__ fm, long fm_stride, float *__restrict__ spat,
            long spat_stride) {
  using C = TsF2<P, Q, R>;
  extern __shared__ __align__(16) float2 ts_smem_f2s[];
  float2 *twq = ts_smem_f2s;
  float2 *b = twq + C::TWQ;
  const long f = blockIdx.y;
  const TsF2Rows<C, false> rows{(int)blockIdx.x * R, ft.nlat, 0};
  ts_f2_twq<C>(twq, ft);
  ts_f2_pack<C>(b, fm + f * fm_stride, ft, rows);
  __syncthreads();
  float *dst = spat + f * spat_stride;
  if ((reinterpret_cast<unsigned long long>(dst) & 15) == 0 && (ft.nphi & 3) == 0 &&
      (C::H & 1) == 0 && ((C::TWQ * sizeof(float2)) & 15) == 0)
    ts_f2_inverse_bulk<C>(b, twq, dst, ft.nphi, rows);
  else
    ts_f2_inverse_out<C>(b, twq, dst, ft.nphi, rows);
}

// spat[field][lat][phi] -> g[field][m][lat].  grid = (ceil(nlat/R), fields).
template <int P, int Q, int R>
__global__ void __launch_bounds__(P *R, TS_F2_MINB(P, R))
ts_f2_analys(TsFftTab ft, const float *__restrict__ spat, long spat_stride,
             float2 *__restrict__ g, long g_stride) {
  using C = TsF2<P, Q, R>;
  extern __shared__ float2 ts_smem_f2a[];
  float2 *twq = ts_smem_f2a;
  float2 *b = twq + C::TWQ;
  const long f = blockIdx.y;
  const TsF2Rows<C, false> rows{(int)blockIdx.x * R, ft.nlat, 0};
  ts_f2_twq<C>(twq, ft);
  __syncthreads();
  ts_f2_forward_in<C>(b, twq, spat + f * spat_stride, ft.nphi, rows);
  ts_f2_unpack<C>(b, g + f * g_stride, ft, rows);
}

// spat[field][lat][phi] -> W image.  grid = (ceil(nh/(R/2)), fields).
template <int P, int Q, int R>
__global__ void __launch_bounds__(P *R, TS_F2_MINB(P, R))
ts_f2_analys_w(TsFftTab ft, const float *__restrict__ spat, long spat_stride,
               const float *__restrict__ wq, char *wimg, int nfb, int fpb, int nlc, int nh,
               const int *__restrict__ w_kmin) {
  using C = TsF2<P, Q, R>;
  extern __shared__ float2 ts_smem_f2w[];
  float2 *twq = ts_smem_f2w;
  float2 *b = twq + C::TWQ;
  const long f = blockIdx.y;
  const int lat0 = blockIdx.x * (R / 2);
  const TsF2Rows<C, true> rows{lat0, ft.nlat, nh};
  ts_f2_twq<C>(twq, ft);
  __syncthreads();
  ts_f2_forward_in<C>(b, twq, spat + f * spat_stride, ft.nphi, rows);
  ts_f2_write_w<C>(b, lat0, f, ft, wq, wimg, nfb, fpb, nlc, nh, w_kmin);
}

// ------------------------------------------------------- fused grid phase
//
// One launch runs a whole grid phase of a compiled model for R latitude rows
// of one instance: the synthesis of the phase's NSYN spectral inputs, the
// generated element-wise program at every grid point (Prog::eval, two points
// per packed complex value), and the analysis of its NANA outputs.  The grid
// values stay in shared memory; a grid variable reaches HBM only when it is
// materialised (NGOUT outputs: a displayed field, or a value a later phase
// reads).  PAIRED (tensor-core plans) takes latitude pairs and writes the
// analysis as the W image, otherwise it writes
//   gm [inst][NANA][mmax+1][nlat].
// grid = (ceil(nlat/R) or ceil(nh/(R/2)), instances), block = P*R; shared
// memory ts_f2_smem_bytes(max(NSYN, NANA, 1)).

// phase 1 of the synthesis for the row blocks at b + s bs (s < NS): Q-point
// DFTs over k2, twiddles, transposed store (two barriers)
template <class C, int NS>
TS_DEV void ts_f2_inv_phase1_n(float2 *b, long bs, const float2 *twq) {
  int r, k1;
  ts_f2_rk<C>(threadIdx.x, r, k1);
  float2 x[NS][C::Q];
#pragma unroll
  for (int s = 0; s < NS; s++) {
    const float2 *row = b + s * bs + r * C::RP;
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) x[s][k2] = row[k1 + C::P * k2];
  }
#pragma unroll
  for (int s = 0; s < NS; s++) ts_dft<C::Q, +1>(x[s]);
#pragma unroll
  for (int n2 = 1; n2 < C::Q; n2++) {
    const float2 t = twq[n2 * C::P1 + k1];
#pragma unroll
    for (int s = 0; s < NS; s++) x[s][n2] = c_mul(x[s][n2], t);
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; s++) {
    float2 *row = b + s * bs + r * C::RP;
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) row[n2 * C::P1 + k1] = x[s][n2];
  }
  __syncthreads();
}

// phase 2 of the analysis for the row blocks at b + s bs (s < NS): Q-point
// DFTs over n2 from the transposed layout, natural store (two barriers)
template <class C, int NS>
TS_DEV void ts_f2_fwd_phase2_n(float2 *b, long bs) {
  int r, k1;
  ts_f2_rk<C>(threadIdx.x, r, k1);
  float2 x[NS][C::Q];
#pragma unroll
  for (int s = 0; s < NS; s++) {
    const float2 *row = b + s * bs + r * C::RP;
#pragma unroll
    for (int n2 = 0; n2 < C::Q; n2++) x[s][n2] = row[n2 * C::P1 + k1];
  }
#pragma unroll
  for (int s = 0; s < NS; s++) ts_dft<C::Q, -1>(x[s]);
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; s++) {
    float2 *row = b + s * bs + r * C::RP;
#pragma unroll
    for (int k2 = 0; k2 < C::Q; k2++) row[k1 + C::P * k2] = x[s][k2];
  }
  __syncthreads();
}

// ts_f2_write_w for NS fields f0 + s (row blocks b + s * bs): every value is
// computed from shared memory first and the stores follow back to back, so
// the reads of one k do not wait behind the stores of the previous one.  A
// thread takes at most (Q + 1) / 2 orders (mmax < H).
template <class C, int NS>
TS_DEV void ts_f2_write_w_n(const float2 *b, long bs, int lat0, long f0, const TsFftTab &ft,
                            const float *__restrict__ wq, char *wimg, int nfb, int fpb, int nlc,
                            int nh, const int *__restrict__ w_kmin) {
  constexpr int NPR = C::R / 2, KS = 2 * C::P, NIT = (C::Q + 1) / 2;
  const int j = threadIdx.x % NPR;
  const int lat = lat0 + j;
  if (lat >= nh) return;
  const bool south = ft.nlat - 1 - lat != lat;
  const float w = 0.5f * __ldg(wq + lat);  // times 2 X[k] of both rows
  // k groups as in ts_f2_write_w (the two halves of a half-warp 8 apart)
  const int g = threadIdx.x / NPR;
  const int k0 = KS % 16 == 0 ? (g & ~15) + ((g & 1) << 3) + ((g >> 1) & 7) : g;
  const int kl0 = w_kmin ? __ldg(w_kmin + 2 * (lat >> 5)) : ft.mmax + 1;
  const int kl1 = w_kmin ? __ldg(w_kmin + 2 * (lat >> 5) + 1) : ft.mmax + 1;
  const int kend = min(ft.mmax + 1, max(kl0, kl1));
  float2 t[NIT];
#pragma unroll
  for (int i = 0; i < NIT; i++)
    t[i] = k0 + KS * i < kend ? __ldg(ft.tw + k0 + KS * i) : make_float2(0.f, 0.f);
  float4 v[NS][NIT];  // w (N + S), w (N - S) of (re, im) per order
#pragma unroll
  for (int s = 0; s < NS; s++) {
    const float2 *rn = b + s * bs + j * C::RP, *rs = b + s * bs + (NPR + j) * C::RP;
#pragma unroll
    for (int i = 0; i < NIT; i++) {
      const int k = k0 + KS * i;
      v[s][i] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (k < kend) {
        const float2 xn = ts_f2_xk2<C>(rn, k, t[i]);
        const float2 xs = south ? ts_f2_xk2<C>(rs, k, t[i]) : make_float2(0.f, 0.f);
        v[s][i] = make_float4(w * (xn.x + xs.x), w * (xn.y + xs.y), w * (xn.x - xs.x),
                              w * (xn.y - xs.y));
      }
    }
  }
  const long kstep = (long)nfb * 2 * nlc * 16384, pstep = (long)nlc * 16384;
#pragma unroll
  for (int s = 0; s < NS; s++) {
    const long f = f0 + s;
    const long fb = f / fpb;
    const int fl = (int)(f - fb * fpb);
    const int o_re = ts_swz_img(2 * fl, lat & 31), o_im = ts_swz_img(2 * fl + 1, lat & 31);
    char *base = wimg + ((long)fb * 2 * nlc + (lat >> 5)) * 16384;
#pragma unroll
    for (int i = 0; i < NIT; i++) {
      const int k = k0 + KS * i;
      char *blk = base + k * kstep;
      if (k < kl0 && k < kend) {
        *reinterpret_cast<float *>(blk + o_re) = v[s][i].x;
        *reinterpret_cast<float *>(blk + o_im) = v[s][i].y;
      }
      if (k < kl1 && k < kend) {
        *reinterpret_cast<float *>(blk + pstep + o_re) = v[s][i].z;
        *reinterpret_cast<float *>(blk + pstep + o_im) = v[s][i].w;
      }
    }
  }
}

// f(TsIC<s0>{}, TsIC<n>{}) for the groups [s0, s0 + n) of at most G of [0, N)
template <int N, int G, int S0 = 0, class F>
TS_DEV void ts_f2_groups(F &&f) {
  if constexpr (S0 < N) {
    f(TsIC<S0>{}, TsIC<(N - S0 < G ? N - S0 : G)>{});
    ts_f2_groups<N, G, S0 + G>(f);
  }
}

// Species go through the synthesis and analysis passes two at a time: one
// pair of barriers and one batch of loads per pair (the registers of two
// P-point rows per thread are what the middle section holds anyway).
template <class Prog, int P, int Q, int R, bool PAIRED>
__global__ void __launch_bounds__(P *R, TS_F2_PHASE_MINB(P, R))
ts_f2_phase(TsFftTab ft, TsPhaseIO io) {
  using C = TsF2<P, Q, R>;
  constexpr int NSYN = Prog::NSYN, NGIN = Prog::NGIN, NANA = Prog::NANA, NGOUT = Prog::NGOUT;
  constexpr int NIN = NSYN + NGIN;
  constexpr int NB = NSYN > NANA ? NSYN : (NANA > 0 ? NANA : 1);
  extern __shared__ float2 ts_smem_f2p[];
  float2 *twq = ts_smem_f2p;
  float2 *buf = twq + C::TWQ;
  constexpr int BS = C::R * C::RP;  // floats2 per row block
  const long inst = blockIdx.y;
  const int lat0 = blockIdx.x * (PAIRED ? R / 2 : R);
  const TsF2Rows<C, PAIRED> rows{lat0, ft.nlat, io.nh};
  ts_f2_twq<C>(twq, ft);
  ts_f2_groups<NSYN, 2>([&](auto s0c, auto nc) {
    constexpr int s0 = decltype(s0c)::value, n = decltype(nc)::value;
    ts_f2_pack_n<C, n>(buf + s0 * BS, BS, io.fm + (inst * NSYN + s0) * io.field, io.field, ft,
                       rows);
  });
  __syncthreads();
  ts_f2_groups<NSYN, 2>([&](auto s0c, auto nc) {
    constexpr int s0 = decltype(s0c)::value, n = decltype(nc)::value;
    ts_f2_inv_phase1_n<C, n>(buf + s0 * BS, BS, twq);
  });

  // Thread (row r, n2) holds, after the synthesis's P-point DFTs, every
  // species at the grid points n = Q n1 + n2 (n1 < P): exactly the inputs
  // of the analysis's first P-point DFTs.  The program runs there, in
  // registers; grid inputs and outputs move as 128-byte runs (16 lanes of
  // consecutive n2).
  if (threadIdx.x < C::Q * C::R) {
    const int r = threadIdx.x / C::Q, n2 = threadIdx.x - r * C::Q;
    const int lat = rows(r);
    const float *prm = io.prm + inst * io.nprm;
    float2 w[NB][P];
#pragma unroll
    for (int s = 0; s < NSYN; s++) {
      const float2 *row = buf + s * BS + r * C::RP + n2 * C::P1;
#pragma unroll
      for (int k1 = 0; k1 < P; k1++) w[s][k1] = row[k1];
      ts_dft<P, +1>(w[s]);
    }
#pragma unroll
    for (int n1 = 0; n1 < P; n1++) {
      const long n = (long)Q * n1 + n2;
      float in0[NIN > 0 ? NIN : 1], in1[NIN > 0 ? NIN : 1];
#pragma unroll
      for (int s = 0; s < NSYN; s++) {
        in0[s] = w[s][n1].x;
        in1[s] = w[s][n1].y;
      }
#pragma unroll
      for (int gi = 0; gi < NGIN; gi++) {
        float2 g = make_float2(0.f, 0.f);
        if (lat >= 0)
          g = reinterpret_cast<const float2 *>(io.gin[gi] + inst * io.gin_stride[gi] +
                                               (long)lat * ft.nphi)[n];
        in0[NSYN + gi] = g.x;
        in1[NSYN + gi] = g.y;
      }
      float out0[NANA + NGOUT > 0 ? NANA + NGOUT : 1], out1[NANA + NGOUT > 0 ? NANA + NGOUT : 1];
      Prog::eval(in0, out0, prm);
      Prog::eval(in1, out1, prm);
#pragma unroll
      for (int o = 0; o < NANA; o++) w[o][n1] = make_float2(out0[o], out1[o]);
      if (lat >= 0) {
#pragma unroll
        for (int o = 0; o < NGOUT; o++)
          reinterpret_cast<float2 *>(io.gout[o] + inst * io.gout_stride[o] +
                                     (long)lat * ft.nphi)[n] = make_float2(out0[NANA + o], out1[NANA + o]);
      }
    }
#pragma unroll
    for (int o = 0; o < NANA; o++) {
      ts_dft<P, -1>(w[o]);
      float2 *row = buf + o * BS + r * C::RP + n2 * C::P1;
      row[0] = w[o][0];
#pragma unroll
      for (int k1 = 1; k1 < P; k1++) row[k1] = c_mul(w[o][k1], c_conj(twq[n2 * C::P1 + k1]));
    }
  }
  __syncthreads();
  ts_f2_groups<NANA, 2>([&](auto s0c, auto nc) {
    constexpr int s0 = decltype(s0c)::value, n = decltype(nc)::value;
    ts_f2_fwd_phase2_n<C, n>(buf + s0 * BS, BS);
  });
  if constexpr (PAIRED) {
    ts_f2_groups<NANA, 2>([&](auto s0c, auto nc) {
      constexpr int s0 = decltype(s0c)::value, n = decltype(nc)::value;
      ts_f2_write_w_n<C, n>(buf + s0 * BS, BS, lat0, inst * NANA + s0, ft, io.wq, io.wimg,
                            io.w_nfb, io.w_fpb, io.w_nlc, io.nh, io.w_kmin);
    });
  } else {
#pragma unroll 1
    for (int k = 0; k < NANA; k++)
      ts_f2_unpack<C>(buf + k * BS, io.gm + (inst * NANA + k) * io.field, ft, rows);
  }
}
