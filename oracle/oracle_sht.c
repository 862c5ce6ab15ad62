/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C, f64 restatement of the reference's CPU ground truth for the
 * spherical-harmonic transform path of turing-sphere, used by the tests, by
 * the smoke check and by the benchmark's CPU-baseline leg as the checker.
 * Nothing in the product library links, calls or loads this file.
 *
 * Each function names the reference file:line it restates (paths are relative
 * to the turing-sphere project root).  Conventions (layout.ts:1-16):
 *   - spectral Q_lm complex, m >= 0 only, interleaved [re, im], m-major order
 *     lm(l, m) = m*(lmax+1) - m*(m-1)/2 + (l - m);
 *   - spatial field real, spat[ilat*nphi + iphi], ilat north -> south;
 *   - orthonormal harmonics with the Condon-Shortley phase;
 *   - analysis carries the 2*pi/nphi longitude quadrature weight.
 *
 * Parity pins: tests/golden holds scipy sph_harm_y / numpy leggauss vectors and
 * outputs of the reference's own bench/shtns/spec.h (compiled from its sources
 * by oracle/Makefile into oracle/_ref/), against which this file is checked.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------- layout.ts */

/* layout.ts:24-27 */
long ors_nlm(int lmax, int mmax) {
  return (long)(mmax + 1) * (lmax + 1) - (long)mmax * (mmax + 1) / 2;
}

/* layout.ts:30-32 */
long ors_lm_index(int lmax, int l, int m) {
  return (long)m * (lmax + 1) - (long)m * (m - 1) / 2 + (l - m);
}

/* layout.ts:34-44.  0 = valid, else 1..4 = which rule failed (lmax, mmax,
 * nlat, nphi), matching the order of the reference's checks. */
int ors_validate(int lmax, int mmax, int nlat, int nphi) {
  if (lmax < 1) return 1;
  if (mmax < 0 || mmax > lmax) return 2;
  if (nlat <= lmax) return 3;
  if (nphi < 2 * mmax + 1) return 4;
  return 0;
}

/* layout.ts:53-59 (dealias rule; nphi rounded up to a power of two) */
void ors_grid_for_lmax(int lmax, int pdeg, int *nlat, int *nphi) {
  double minlat = ((double)(pdeg + 1) * lmax + 1) / 2.0;
  if (minlat < lmax + 1) minlat = lmax + 1;
  *nlat = 2 * (int)ceil(minlat / 2.0);
  int n = 1;
  while (n < (pdeg + 1) * lmax + 1) n *= 2;
  *nphi = n;
}

/* -------------------------------------------------------------- gauss.ts */

/* gauss.ts:11-51: Newton on P_n, nodes x = cos(theta) in decreasing order. */
void ors_gauss(int n, double *x, double *w) {
  int half = (n + 1) >> 1;
  for (int i = 0; i < half; i++) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int iter = 0; iter < 100; iter++) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; j++) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (fabs(dz) < 1e-15 * fabs(z) + 1e-300) {
        double q1 = 1.0, q2 = 0.0;
        for (int j = 1; j <= n; j++) {
          double q3 = q2;
          q2 = q1;
          q1 = ((2.0 * j - 1.0) * z * q2 - (j - 1.0) * q3) / j;
        }
        pp = n * (z * q1 - q2) / (z * z - 1.0);
        z -= q1 / pp;
        break;
      }
    }
    x[i] = z;
    x[n - 1 - i] = -z;
    double wi = 2.0 / ((1.0 - z * z) * pp * pp);
    w[i] = wi;
    w[n - 1 - i] = wi;
  }
  if (n & 1) x[half - 1] = 0.0;
}

/* ------------------------------------------------------------- coeffs.ts */

/* coeffs.ts:28-56.  amm[mmax+1]; ab[2*nlm] = (a_l^m, b_l^m) per lm. */
void ors_legendre_coeffs(int lmax, int mmax, double *amm, double *ab) {
  long nlm = ors_nlm(lmax, mmax);
  memset(ab, 0, sizeof(double) * 2 * nlm);
  double t = 1.0 / (4.0 * M_PI);
  amm[0] = sqrt(t);
  for (int m = 1; m <= mmax; m++) {
    t *= (2.0 * m + 1.0) / (2.0 * m);
    amm[m] = -sqrt(t);
    if (m % 2 == 0) amm[m] = -amm[m];
  }
  for (int m = 0; m <= mmax; m++) {
    if (m + 1 <= lmax) {
      long lm = ors_lm_index(lmax, m + 1, m);
      ab[2 * lm] = sqrt(2.0 * m + 3.0);
      ab[2 * lm + 1] = 0.0;
    }
    for (int l = m + 2; l <= lmax; l++) {
      long lm = ors_lm_index(lmax, l, m);
      double t1 = (double)(l + m) * (l - m);
      double t2 = (double)(l - 1 + m) * (l - 1 - m);
      ab[2 * lm] = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / t1);
      ab[2 * lm + 1] = -sqrt((2.0 * l + 1.0) / (2.0 * l - 3.0) * (t2 / t1));
    }
  }
}

/* coeffs.ts:64-85: ytilde_l^m(theta) for l = m..lmax at one point, plain f64
 * recurrence.  out has lmax-m+1 entries. */
void ors_legendre_row(const double *amm, const double *ab, int lmax, int m, double ct,
                      double st, double *out) {
  double y0 = amm[m] * pow(st, m);
  out[0] = y0;
  if (m == lmax) return;
  long base = ors_lm_index(lmax, m, m);
  double y1 = ab[2 * (base + 1)] * ct * y0;
  out[1] = y1;
  for (int l = m + 2; l <= lmax; l++) {
    long lm = base + (l - m);
    double y2 = ab[2 * lm] * ct * y1 + ab[2 * lm + 1] * y0;
    y0 = y1;
    y1 = y2;
    out[l - m] = y2;
  }
}

/* ---------------------------------------------------------- reference.ts */

typedef struct {
  int lmax, mmax, nlat, nphi;
  long nlm;
  double *ct, *st, *wg, *amm, *ab;
  double *cosk, *sink; /* (cos, sin)(2*pi*k/nphi), k < nphi, in f64 */
} ors_plan;

/* reference.ts:20-35 (constructor) */
ors_plan *ors_plan_create(int lmax, int mmax, int nlat, int nphi) {
  if (ors_validate(lmax, mmax, nlat, nphi) != 0) return NULL;
  ors_plan *p = (ors_plan *)calloc(1, sizeof(ors_plan));
  p->lmax = lmax;
  p->mmax = mmax;
  p->nlat = nlat;
  p->nphi = nphi;
  p->nlm = ors_nlm(lmax, mmax);
  p->ct = (double *)malloc(sizeof(double) * nlat);
  p->st = (double *)malloc(sizeof(double) * nlat);
  p->wg = (double *)malloc(sizeof(double) * nlat);
  p->amm = (double *)malloc(sizeof(double) * (mmax + 1));
  p->ab = (double *)malloc(sizeof(double) * 2 * p->nlm);
  p->cosk = (double *)malloc(sizeof(double) * nphi);
  p->sink = (double *)malloc(sizeof(double) * nphi);
  ors_gauss(nlat, p->ct, p->wg);
  for (int i = 0; i < nlat; i++) p->st[i] = sqrt(1.0 - p->ct[i] * p->ct[i]);
  ors_legendre_coeffs(lmax, mmax, p->amm, p->ab);
  for (int k = 0; k < nphi; k++) {
    double phi = 2.0 * M_PI * k / nphi;
    p->cosk[k] = cos(phi);
    p->sink[k] = sin(phi);
  }
  return p;
}

void ors_plan_destroy(ors_plan *p) {
  if (!p) return;
  free(p->ct);
  free(p->st);
  free(p->wg);
  free(p->amm);
  free(p->ab);
  free(p->cosk);
  free(p->sink);
  free(p);
}

void ors_plan_nodes(const ors_plan *p, double *ct, double *wg) {
  memcpy(ct, p->ct, sizeof(double) * p->nlat);
  memcpy(wg, p->wg, sizeof(double) * p->nlat);
}

/* threads > 0: that many OpenMP threads; 0: every host core (set each call,
 * so a single-threaded call does not leave later calls on one thread). */
static void ors_set_threads(int threads) {
#ifdef _OPENMP
  omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs());
#else
  (void)threads;
#endif
}

/* reference.ts:41-61: F_m(theta_i) = sum_l Q_lm ytilde_l^m(theta_i),
 * fm[2*(m*nlat + i) + {0,1}]. */
void ors_legendre_synth(const ors_plan *p, const double *qlm, double *fm, int threads) {
  ors_set_threads(threads);
  const int lmax = p->lmax, mmax = p->mmax, nlat = p->nlat;
#pragma omp parallel
  {
    double *row = (double *)malloc(sizeof(double) * (lmax + 1));
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < nlat; i++) {
      for (int m = 0; m <= mmax; m++) {
        ors_legendre_row(p->amm, p->ab, lmax, m, p->ct[i], p->st[i], row);
        double re = 0, im = 0;
        long base = ors_lm_index(lmax, m, m);
        for (int l = m; l <= lmax; l++) {
          double y = row[l - m];
          re += y * qlm[2 * (base + l - m)];
          im += y * qlm[2 * (base + l - m) + 1];
        }
        long o = 2L * ((long)m * nlat + i);
        fm[o] = re;
        fm[o + 1] = im;
      }
    }
    free(row);
  }
}

/* reference.ts:64-84: spat[i*nphi + j] = Re F_0 + 2 sum_{m>=1} Re(F_m e^{i m phi_j}).
 * The phase uses an f64 table at (m*j mod nphi), the exact angle the
 * reference's cos(m*phi) evaluates (to the last bit of f64). */
void ors_fourier_synth(const ors_plan *p, const double *fm, double *spat, int threads) {
  ors_set_threads(threads);
  const int mmax = p->mmax, nlat = p->nlat, nphi = p->nphi;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nlat; i++) {
    for (int j = 0; j < nphi; j++) {
      double v = fm[2L * i];
      long idx = 0;
      for (int m = 1; m <= mmax; m++) {
        idx += j;
        if (idx >= nphi) idx -= nphi;
        long o = 2L * ((long)m * nlat + i);
        v += 2.0 * (fm[o] * p->cosk[idx] - fm[o + 1] * p->sink[idx]);
      }
      spat[(long)i * nphi + j] = v;
    }
  }
}

void ors_synth(const ors_plan *p, const double *qlm, double *spat, int threads) {
  double *fm = (double *)malloc(sizeof(double) * 2 * (p->mmax + 1) * (long)p->nlat);
  ors_legendre_synth(p, qlm, fm, threads);
  ors_fourier_synth(p, fm, spat, threads);
  free(fm);
}

/* reference.ts:90-104: G_m(theta_i) = (2 pi / nphi) sum_j f_ij e^{-i m phi_j} */
void ors_fourier_analys(const ors_plan *p, const double *spat, double *gm, int threads) {
  ors_set_threads(threads);
  const int mmax = p->mmax, nlat = p->nlat, nphi = p->nphi;
  const double norm = 2.0 * M_PI / nphi;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nlat; i++) {
    for (int m = 0; m <= mmax; m++) {
      double re = 0, im = 0;
      long idx = 0;
      for (int j = 0; j < nphi; j++) {
        double f = spat[(long)i * nphi + j];
        re += f * p->cosk[idx];
        im -= f * p->sink[idx];
        idx += m;
        if (idx >= nphi) idx -= nphi;
      }
      long o = 2L * ((long)m * nlat + i);
      gm[o] = re * norm;
      gm[o + 1] = im * norm;
    }
  }
}

/* reference.ts:105-117: Q_lm = sum_i w_i ytilde_l^m(theta_i) G_m(theta_i) */
void ors_legendre_analys(const ors_plan *p, const double *gm, double *qlm, int threads) {
  ors_set_threads(threads);
  const int lmax = p->lmax, mmax = p->mmax, nlat = p->nlat;
  memset(qlm, 0, sizeof(double) * 2 * p->nlm);
#pragma omp parallel
  {
    double *row = (double *)malloc(sizeof(double) * (lmax + 1));
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= mmax; m++) {
      long base = ors_lm_index(lmax, m, m);
      for (int i = 0; i < nlat; i++) {
        ors_legendre_row(p->amm, p->ab, lmax, m, p->ct[i], p->st[i], row);
        long o = 2L * ((long)m * nlat + i);
        double wr = p->wg[i] * gm[o];
        double wi = p->wg[i] * gm[o + 1];
        for (int l = m; l <= lmax; l++) {
          double y = row[l - m];
          qlm[2 * (base + l - m)] += y * wr;
          qlm[2 * (base + l - m) + 1] += y * wi;
        }
      }
    }
    free(row);
  }
}

void ors_analys(const ors_plan *p, const double *spat, double *qlm, int threads) {
  double *gm = (double *)malloc(sizeof(double) * 2 * (p->mmax + 1) * (long)p->nlat);
  ors_fourier_analys(p, spat, gm, threads);
  ors_legendre_analys(p, gm, qlm, threads);
  free(gm);
}

/* ------------------------------------------------------------ seeding */

/* reference.ts:122-136: xorshift32 spectrum in [-1, 1), rounded to float,
 * m = 0 imaginary parts zeroed. */
void ors_random_spectrum(int lmax, int mmax, uint32_t seed, float *q) {
  long nlm = ors_nlm(lmax, mmax);
  uint32_t s = seed;
  for (long k = 0; k < 2 * nlm; k++) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    q[k] = (float)(((double)s / 4294967296.0) * 2.0 - 1.0);
  }
  for (int l = 0; l <= lmax; l++) q[2 * ors_lm_index(lmax, l, 0) + 1] = 0.0f;
}

/* noise.ts:15-24: mulberry32, uniform in [0, 1). */
typedef struct {
  uint32_t s;
  int have_spare;
  double spare;
} ors_rng;

void ors_rng_init(ors_rng *r, uint32_t seed) {
  r->s = seed;
  r->have_spare = 0;
  r->spare = 0.0;
}

double ors_rand(ors_rng *r) {
  r->s += 0x6d2b79f5u;
  uint32_t t = r->s;
  t = (t ^ (t >> 15)) * (t | 1u);
  t ^= t + (t ^ (t >> 7)) * (t | 61u);
  return (double)(t ^ (t >> 14)) / 4294967296.0;
}

/* noise.ts:27-43: Box-Muller with a spare. */
double ors_randn(ors_rng *r) {
  if (r->have_spare) {
    r->have_spare = 0;
    return r->spare;
  }
  double u = 0.0;
  while (u == 0.0) u = ors_rand(r);
  double rad = sqrt(-2.0 * log(u));
  double th = 2.0 * M_PI * ors_rand(r);
  r->spare = rad * sin(th);
  r->have_spare = 1;
  return rad * cos(th);
}

/* noise.ts:46-51: amp-scaled normals per grid point, stored as float. */
void ors_seeded_noise(long npts, double amp, uint32_t seed, float *out) {
  ors_rng r;
  ors_rng_init(&r, seed);
  for (long i = 0; i < npts; i++) out[i] = (float)(amp * ors_randn(&r));
}

/* bench-sht.ts:132-144: mulberry32 spectrum in [-1, 1), m = 0 imag zeroed. */
void ors_seeded_spectrum(int lmax, int mmax, uint32_t seed, float *q) {
  ors_rng r;
  ors_rng_init(&r, seed);
  long lm = 0;
  for (int m = 0; m <= mmax; m++)
    for (int l = m; l <= lmax; l++, lm++) {
      q[2 * lm] = (float)(2.0 * ors_rand(&r) - 1.0);
      float im = (float)(2.0 * ors_rand(&r) - 1.0);
      q[2 * lm + 1] = (m == 0) ? 0.0f : im;
    }
}

/* model.ts:46-56: lam = l(l+1), duplicated over re/im. */
void ors_eigenvalues(int lmax, int mmax, double *lam) {
  for (int m = 0; m <= mmax; m++)
    for (int l = m; l <= lmax; l++) {
      long i = ors_lm_index(lmax, l, m);
      lam[2 * i] = (double)l * (l + 1);
      lam[2 * i + 1] = (double)l * (l + 1);
    }
}

/* ------------------------------------------------------------ model steps
 *
 * The `step` functions of the reference models, in f64, with the .m's
 * operation order: synth every species, the reaction on the grid, analys
 * every reaction output, then the IMEX update with (dt*D) formed as one
 * product (spec.h:394-408).  `u.^3` is u*u*u (wgsl.ts:224-257).
 *
 *  model 0 schnakenberg.m:23-29   params (a, b, D1, D2, dt)
 *  model 1 brusselator.m:22-28    params (A, B, D1, D2, dt)
 *  model 2 allencahn.m:19-22      params (eps2, dt)
 *  model 3 test/models/linear.m   params (c, D, dt)
 *  model 4 test/models/logistic.m params (r, D, dt)
 */
int ors_model_species(int model) { return (model == 0 || model == 1) ? 2 : 1; }

static void ors_react(int model, const double *prm, double u, double v, double *r1,
                      double *r2) {
  switch (model) {
    case 0: {
      double uuv = u * u * v;
      *r1 = prm[0] - u + uuv;
      *r2 = prm[1] - uuv;
      break;
    }
    case 1: {
      double uuv = u * u * v;
      *r1 = prm[0] - (prm[1] + 1.0) * u + uuv;
      *r2 = prm[1] * u - uuv;
      break;
    }
    case 2:
      *r1 = u - u * u * u;
      break;
    case 3:
      *r1 = prm[0] * u;
      break;
    case 4:
      *r1 = prm[0] * u * (1.0 - u);
      break;
  }
}

/* state: S species x 2*nlm, advanced in place by nsteps. */
int ors_model_step(const ors_plan *p, int model, const double *prm, double *state, int nsteps,
                   int threads) {
  const int S = ors_model_species(model);
  const long nlm = p->nlm;
  const long npts = (long)p->nlat * p->nphi;
  double dt, dtD[2] = {0, 0};
  switch (model) {
    case 0:
    case 1:
      dt = prm[4];
      dtD[0] = dt * prm[2];
      dtD[1] = dt * prm[3];
      break;
    case 2:
      dt = prm[1];
      dtD[0] = dt * prm[0];
      break;
    case 3:
    case 4:
      dt = prm[2];
      dtD[0] = dt * prm[1];
      break;
    default:
      return -1;
  }
  double *lam = (double *)malloc(sizeof(double) * 2 * nlm);
  ors_eigenvalues(p->lmax, p->mmax, lam);
  double *grid = (double *)malloc(sizeof(double) * S * npts);
  double *rgrid = (double *)malloc(sizeof(double) * S * npts);
  double *rq = (double *)malloc(sizeof(double) * 2 * nlm);
  for (int s = 0; s < nsteps; s++) {
    for (int k = 0; k < S; k++) ors_synth(p, state + k * 2 * nlm, grid + k * npts, threads);
    for (long i = 0; i < npts; i++) {
      double r1 = 0, r2 = 0;
      ors_react(model, prm, grid[i], S > 1 ? grid[npts + i] : 0.0, &r1, &r2);
      rgrid[i] = r1;
      if (S > 1) rgrid[npts + i] = r2;
    }
    for (int k = 0; k < S; k++) {
      ors_analys(p, rgrid + k * npts, rq, threads);
      double *U = state + k * 2 * nlm;
      for (long i = 0; i < 2 * nlm; i++) U[i] = (U[i] + dt * rq[i]) / (1.0 + dtD[k] * lam[i]);
    }
  }
  free(lam);
  free(grid);
  free(rgrid);
  free(rq);
  return 0;
}

/* ---------------------------------------------------------------- adjoint
 *
 * The reference has no differentiation.  These are the f64 transposes of this
 * file's own forward step, the check for a GPU adjoint: each function is the
 * exact adjoint (transpose) of the f64 map above it applies to.
 *
 * Transforms.  Reading coefficients as 2*nlm reals and the grid as
 * nlat*nphi reals, ors_synth is S and ors_analys is A with
 *   S[(i,j),(l,m,re)] =  c_m P_lm(x_i) cos(m phi_j),
 *   S[(i,j),(l,m,im)] = -c_m P_lm(x_i) sin(m phi_j),
 *   A[(l,m,.),(i,j)]  = w'_i S[(i,j),(l,m,.)] / c_m,
 * c_0 = 1, c_m = 2 (m >= 1), w'_i = w_i 2 pi/nphi (the Gauss weight times
 * the longitude quadrature weight).  Hence S^T = C A W'^-1 and
 * A^T = W' S C^-1; the m = 0 imaginary entries are zero rows of A and zero
 * columns of S, so both adjoints leave them zero. */

static double ors_cm(int lmax, long lm) {
  /* m of coefficient lm: m = 0 occupies lm = 0..lmax */
  return lm <= lmax ? 1.0 : 2.0;
}

/* qbar = S^T gbar */
void ors_synth_adjoint(const ors_plan *p, const double *gbar, double *qbar, int threads) {
  const long npts = (long)p->nlat * p->nphi;
  double *g = (double *)malloc(sizeof(double) * npts);
  const double lon = 2.0 * M_PI / p->nphi;
  for (int i = 0; i < p->nlat; i++)
    for (int j = 0; j < p->nphi; j++) {
      long o = (long)i * p->nphi + j;
      g[o] = gbar[o] / (p->wg[i] * lon);
    }
  ors_analys(p, g, qbar, threads);
  for (long lm = 0; lm < p->nlm; lm++) {
    double c = ors_cm(p->lmax, lm);
    qbar[2 * lm] *= c;
    qbar[2 * lm + 1] = lm <= p->lmax ? 0.0 : qbar[2 * lm + 1] * c;
  }
  free(g);
}

/* gbar = A^T qbar */
void ors_analys_adjoint(const ors_plan *p, const double *qbar, double *gbar, int threads) {
  double *q = (double *)malloc(sizeof(double) * 2 * p->nlm);
  for (long lm = 0; lm < p->nlm; lm++) {
    double c = ors_cm(p->lmax, lm);
    q[2 * lm] = qbar[2 * lm] / c;
    q[2 * lm + 1] = lm <= p->lmax ? 0.0 : qbar[2 * lm + 1] / c;
  }
  ors_synth(p, q, gbar, threads);
  const double lon = 2.0 * M_PI / p->nphi;
  for (int i = 0; i < p->nlat; i++)
    for (int j = 0; j < p->nphi; j++) gbar[(long)i * p->nphi + j] *= p->wg[i] * lon;
  free(q);
}

/* Pointwise vector-Jacobian product of the reaction of ors_react: given the
 * cotangents (r1b, r2b) of its outputs at one grid point, accumulate the
 * cotangents of its inputs (u, v) and of its parameters (pb, in the model's
 * parameter order). */
static void ors_react_vjp(int model, const double *prm, double u, double v, double r1b,
                          double r2b, double *ub, double *vb, double *pb) {
  switch (model) {
    case 0: /* r1 = a - u + u^2 v, r2 = b - u^2 v */
      *ub = (-1.0 + 2.0 * u * v) * r1b - 2.0 * u * v * r2b;
      *vb = u * u * (r1b - r2b);
      pb[0] += r1b;
      pb[1] += r2b;
      break;
    case 1: /* r1 = A - (B+1) u + u^2 v, r2 = B u - u^2 v */
      *ub = (-(prm[1] + 1.0) + 2.0 * u * v) * r1b + (prm[1] - 2.0 * u * v) * r2b;
      *vb = u * u * (r1b - r2b);
      pb[0] += r1b;
      pb[1] += u * (r2b - r1b);
      break;
    case 2: /* r = u - u^3 */
      *ub = (1.0 - 3.0 * u * u) * r1b;
      break;
    case 3: /* r = c u */
      *ub = prm[0] * r1b;
      pb[0] += u * r1b;
      break;
    case 4: /* r = r u (1 - u) */
      *ub = prm[0] * (1.0 - 2.0 * u) * r1b;
      pb[0] += u * (1.0 - u) * r1b;
      break;
  }
}

/* parameter indices of dt and of the diffusion coefficient of each species */
static int ors_imex_indices(int model, int *idt, int *iD) {
  switch (model) {
    case 0:
    case 1:
      *idt = 4;
      iD[0] = 2;
      iD[1] = 3;
      return 2;
    case 2:
      *idt = 1;
      iD[0] = 0;
      return 0;
    case 3:
    case 4:
      *idt = 2;
      iD[0] = 1;
      return 0;
  }
  return -1;
}

/* Reverse mode of `nsteps` steps of ors_model_step from state0 (S x 2 nlm):
 * given final_bar = dL/d(final state), writes init_bar = dL/d(state0) and
 * param_bar = dL/d(params) (the model's parameter order; dt and the
 * diffusion coefficients include their appearance in the implicit solve).
 * States are kept every `every` steps and each segment is recomputed from its
 * checkpoint before it is reversed.  Per step, with d = 1/(1 + dt D lam),
 * U' = (U + dt R) d:
 *   dL/dU += d Ubar',   Rbar = dt d Ubar',   rbar = A^T Rbar (grid),
 *   (ubar, vbar, pbar) += reaction VJP of rbar,  dL/dU += S^T ubar,
 *   dL/d dt += sum d Ubar' (R - D lam U'),  dL/dD += sum -dt lam d U' Ubar'. */
int ors_model_adjoint(const ors_plan *p, int model, const double *prm, const double *state0,
                      int nsteps, int every, const double *final_bar, double *init_bar,
                      double *param_bar, int threads) {
  int idt, iD[2] = {0, 0};
  if (ors_imex_indices(model, &idt, iD) < 0) return -1;
  if (every < 1) every = 1;
  const int S = ors_model_species(model);
  const long n2 = 2 * p->nlm, npts = (long)p->nlat * p->nphi;
  const int nprm = model <= 1 ? 5 : (model == 2 ? 2 : 3);
  const double dt = prm[idt];
  const int nck = (nsteps + every - 1) / every;
  double *ck = (double *)malloc(sizeof(double) * (nck + 1) * S * n2);
  double *seg = (double *)malloc(sizeof(double) * (every + 1) * S * n2);
  double *lam = (double *)malloc(sizeof(double) * n2);
  double *grid = (double *)malloc(sizeof(double) * S * npts);
  double *rgrid = (double *)malloc(sizeof(double) * S * npts);
  double *gbar = (double *)malloc(sizeof(double) * S * npts);
  double *rq = (double *)malloc(sizeof(double) * S * n2);
  double *xbar = (double *)malloc(sizeof(double) * S * n2);
  double *nbar = (double *)malloc(sizeof(double) * S * n2);
  double *tmp = (double *)malloc(sizeof(double) * n2);
  ors_eigenvalues(p->lmax, p->mmax, lam);
  /* forward: checkpoints at steps 0, every, 2 every, ... */
  memcpy(ck, state0, sizeof(double) * S * n2);
  for (int c = 1; c <= nck; c++) {
    memcpy(ck + (long)c * S * n2, ck + (long)(c - 1) * S * n2, sizeof(double) * S * n2);
    int len = (c * every <= nsteps) ? every : nsteps - (c - 1) * every;
    ors_model_step(p, model, prm, ck + (long)c * S * n2, len, threads);
  }
  memcpy(xbar, final_bar, sizeof(double) * S * n2);
  for (int k = 0; k < nprm; k++) param_bar[k] = 0.0;
  for (int c = nck - 1; c >= 0; c--) {
    const int len = ((c + 1) * every <= nsteps) ? every : nsteps - c * every;
    memcpy(seg, ck + (long)c * S * n2, sizeof(double) * S * n2);
    for (int t = 1; t <= len; t++) {
      memcpy(seg + (long)t * S * n2, seg + (long)(t - 1) * S * n2, sizeof(double) * S * n2);
      ors_model_step(p, model, prm, seg + (long)t * S * n2, 1, threads);
    }
    for (int t = len - 1; t >= 0; t--) {
      const double *U = seg + (long)t * S * n2, *Un = seg + (long)(t + 1) * S * n2;
      for (int k = 0; k < S; k++) ors_synth(p, U + k * n2, grid + k * npts, threads);
      for (long i = 0; i < npts; i++) {
        double r1 = 0, r2 = 0;
        ors_react(model, prm, grid[i], S > 1 ? grid[npts + i] : 0.0, &r1, &r2);
        rgrid[i] = r1;
        if (S > 1) rgrid[npts + i] = r2;
      }
      for (int k = 0; k < S; k++) {
        ors_analys(p, rgrid + k * npts, rq + k * n2, threads);
        const double D = prm[iD[k]];
        for (long i = 0; i < n2; i++) {
          const double d = 1.0 / (1.0 + dt * D * lam[i]);
          const double ub = xbar[k * n2 + i];
          param_bar[idt] += ub * d * (rq[k * n2 + i] - D * lam[i] * Un[k * n2 + i]);
          param_bar[iD[k]] += -ub * dt * lam[i] * d * Un[k * n2 + i];
          nbar[k * n2 + i] = ub * d;
          tmp[i] = dt * ub * d;
        }
        ors_analys_adjoint(p, tmp, rgrid + k * npts, threads); /* rgrid now holds rbar */
      }
      for (long i = 0; i < npts; i++) {
        double ub = 0, vb = 0;
        ors_react_vjp(model, prm, grid[i], S > 1 ? grid[npts + i] : 0.0, rgrid[i],
                      S > 1 ? rgrid[npts + i] : 0.0, &ub, &vb, param_bar);
        gbar[i] = ub;
        if (S > 1) gbar[npts + i] = vb;
      }
      for (int k = 0; k < S; k++) {
        ors_synth_adjoint(p, gbar + k * npts, tmp, threads);
        for (long i = 0; i < n2; i++) nbar[k * n2 + i] += tmp[i];
      }
      memcpy(xbar, nbar, sizeof(double) * S * n2);
    }
  }
  memcpy(init_bar, xbar, sizeof(double) * S * n2);
  free(ck);
  free(seg);
  free(lam);
  free(grid);
  free(rgrid);
  free(gbar);
  free(rq);
  free(xbar);
  free(nbar);
  free(tmp);
  return 0;
}
