// Shared device helpers for the turing-sphere SHT kernels.
//
// Every header under kernels/ is compiled twice: by nvcc into the library
// (standalone transforms) and by NVRTC at model-compile time together with
// the generated reaction / IMEX code.  So: no #include of system headers, no
// std::, only CUDA builtins.
#pragma once

#define TS_DEV __device__ __forceinline__

// fp32 extended-range recurrence constants (common.ts:17-20 of the
// reference: SCALE = 2^56, ACCURACY = 1e-15, rescale threshold
// ACCURACY*SCALE + 1).  A per-latitude integer exponent `ny` counts the
// factors of SCALE carried by the running Legendre value; a term contributes
// only once ny == 0.
#define TS_SCALE 72057594037927936.0f
#define TS_INV_SCALE 1.387778780781445675529539585113525390625e-17f
#define TS_ACCURACY 1e-15f
#define TS_RESCALE_THR (TS_ACCURACY * TS_SCALE + 1.0f)

// a >= b ? x : y (derivatives of max/min in generated adjoint code)
TS_DEV float ts_ge_sel(float a, float b, float x, float y) { return a >= b ? x : y; }

TS_DEV float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
TS_DEV float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
TS_DEV float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
TS_DEV float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
TS_DEV float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by +i / -i
TS_DEV float2 c_mul_i(float2 a) { return make_float2(-a.y, a.x); }
TS_DEV float2 c_mul_negi(float2 a) { return make_float2(a.y, -a.x); }

// lm index of (l = m, m) in m-major order (layout.ts:30-32).
TS_DEV long ts_lm_base(int lmax, int m) {
  return (long)m * (lmax + 1) - ((long)m * (m - 1)) / 2;
}

// sin(theta)^m with an extended exponent: returns y and ny such that the
// value is y * SCALE^ny (ny <= 0), y kept above ~ACCURACY.  Binary
// exponentiation over the bits of m; the running power s = st^(2^k) carries
// its own exponent ns and is renormalised whenever it drops below 1/SCALE.
TS_DEV void ts_sinpow(float st, int m, float &y, int &ny) {
  y = 1.0f;
  ny = 0;
  float s = st;
  int ns = 0;
  int bits = m;
  while (bits) {
    if (bits & 1) {
      y *= s;
      ny += ns;
      if (y < TS_ACCURACY + TS_INV_SCALE) {
        y *= TS_SCALE;
        ny -= 1;
      }
    }
    bits >>= 1;
    if (!bits) break;
    s *= s;
    ns += ns;
    if (s < TS_INV_SCALE) {
      s *= TS_SCALE;
      ns -= 1;
    }
  }
}

// Read-only parameters of one transform plan as the kernels see them.
struct TsLegTab {
  const float *ct;   // cos(theta) of the northern latitudes (nh entries)
  const float *st;   // sin(theta)
  const float *wq;   // Gauss weight * 2*pi/nphi
  const float2 *ab;  // (a_l^m, b_l^m) per lm
  const float *amm;  // seed amplitude per m (Condon-Shortley sign included)
  int lmax, mmax, nlat, nh;  // nh = ceil(nlat/2): latitudes a recurrence walks
};

// byte offset of element (row r, k) in a K-major 128B-swizzled tile of
// 32-float rows: 8-row groups of 1024 bytes, 16-byte chunk index XOR row % 8
TS_DEV int ts_swz_img(int r, int k) {
  return (r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 2) ^ (r & 7))) << 4) + ((k & 3) << 2);
}

// A set of coefficient fields read by the Legendre synthesis: field f is
// species s = f % nper of instance i = f / nper, at base[s] + i*inst_stride[s].
#define TS_MAXIO 8
struct TsFields {
  const float2 *base[TS_MAXIO];
  long inst_stride[TS_MAXIO];
  int nper;
};

TS_DEV const float2 *ts_field(const TsFields &q, int f) {
  const int s = f % q.nper;
  return q.base[s] + (long)(f / q.nper) * q.inst_stride[s];
}

struct TsFftTab {
  const float2 *tw;  // (cos, sin)(2*pi*k/nphi), k < nphi
  int nphi, H, mmax, nlat;
  int nst;           // Stockham stages of the H-point complex FFT
  int radix[16];
};

// Tensor-core Legendre tables of a plan (see leg_tc.cuh).
struct TsTcTab {
  const char *synth;        // synthesis image
  const long *synth_off;    // byte offset of each m's block, mmax+1 entries
  const char *anal;         // analysis image
  const long *anal_off;
  int NL, nLT;              // synthesis latitude tile (N of the MMA) and tile count
  int LTL;                  // analysis l-tile (per parity), <= 128
  int nLC;                  // analysis latitude chunks of 32
  int *err;                 // set to 1 when a bounded wait gives up
  const int *chunk_prefix;  // synthesis k-chunks (both parities) before m, mmax+2 entries
  const int *chunk_m;       // chunk -> m
  const int *chunk_pc;      // chunk -> (parity << 16) | chunk-of-parity
  int nchunks;
  unsigned wait_limit;      // polls before a bounded wait gives up (0: the default)
  int stall_copies;         // test hook: the copy warp issues nothing, every wait runs out
  // Polar skip (null: none).  syn_zero[m nLT + lt] = 1 when every table value
  // of synthesis tile (m, lt) is below the skip threshold (the tile's output
  // is written as zeros); ana_c0[(2 m + par) ntile + ltile] = leading latitude
  // chunks of an analysis tile whose table values are all below it (skipped).
  const unsigned char *syn_zero;
  const unsigned char *syn_cs;  // leading degree-chunk pairs of tile (m, lt) left out
  const int *ana_c0;
  int ntile;
};

// The data operands of the tensor-core Legendre stage, kept in HBM as raw fp32
// in the shared-memory byte image the MMA reads (16 KB blocks: 128 rows =
// 64 fields x re|im, 32 k, K-major 128-byte swizzle):
//   q: synthesis, block (chunk_prefix[m] + chunk, field block), k -> l
//   w: analysis, block ((m*w_nfb + field block)*2 + parity)*nLC + latitude
//      chunk, k -> northern latitude, value w*(G_north +- G_south)
struct TsTcImg {
  char *q;
  int q_nfb;
  char *w;
  int w_nfb, w_fpb;  // field blocks and fields per block (<= 64) of w
};

// Grid-phase I/O of a compiled model (see ts_fourier_phase in fourier.cuh).
struct TsPhaseIO {
  const float2 *fm;
  float2 *gm;
  long field;  // (mmax+1)*nlat complex values per field
  const float *gin[TS_MAXIO];
  long gin_stride[TS_MAXIO];  // per instance (0 = shared by all instances)
  float *gout[TS_MAXIO];
  long gout_stride[TS_MAXIO];
  const float *prm;
  int nprm;
  // tensor-core plans: the analysis outputs go to the W image instead of gm
  char *wimg;
  int w_nfb, w_fpb, w_nlc, nh;
  const float *wq;
  const int *w_kmin;  // polar skip of W-image writes (see ts_f2_write_w; null: none)
};

// I/O of a model's generated adjoint kernels: the forward ("tape") kernel of
// an element-wise statement reads its inputs in[] and writes out; the
// reverse kernel reads the inputs and the output cotangent gout, adds the
// input cotangents into gin[] and the parameter gradients into pbar
// ([instance][nprm], double).  Strides are per instance (0 = shared).
struct TsAdjIO {
  const float *in[TS_MAXIO];
  long in_stride[TS_MAXIO];
  float *out;
  long out_stride;
  const float *gout;
  long gout_stride;
  float *gin[TS_MAXIO];
  long gin_stride[TS_MAXIO];
  const float *prm;
  int nprm;
  double *pbar;
  long n;  // elements per instance
};

// Spectral-side I/O of a compiled model's generated code: inputs and outputs
// are [instance][2*nlm] float arrays (instance stride 0 = shared by all).
struct TsSpecIO {
  const float *sin[TS_MAXIO];
  long sin_stride[TS_MAXIO];
  float *sout[TS_MAXIO];
  long sout_stride[TS_MAXIO];
  const float *prm;
  int nprm;
  long n;  // 2*nlm
};

// x^k by repeated multiplication, left to right (x.^k with a literal integer
// exponent; a general pow() is undefined for a negative base).
TS_DEV float ts_pow_i1(float x) { return x; }
TS_DEV float ts_pow_i2(float x) { return x * x; }
TS_DEV float ts_pow_i3(float x) { return x * x * x; }
TS_DEV float ts_pow_i4(float x) { return x * x * x * x; }
TS_DEV float ts_pow_i5(float x) { return x * x * x * x * x; }
TS_DEV float ts_pow_i6(float x) { return x * x * x * x * x * x; }
TS_DEV float ts_pow_i7(float x) { return x * x * x * x * x * x * x; }
TS_DEV float ts_pow_i8(float x) { return x * x * x * x * x * x * x * x; }
TS_DEV float ts_sign(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
