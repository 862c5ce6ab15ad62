/*
 * ORACLE — test infrastructure only.
 *
 * A C-ABI shim over the reference's own native spec header
 * (bench/shtns/spec.h), compiled from where it lies in the reference tree by
 * oracle/Makefile into oracle/_ref/libshtb_spec.so.  It exposes the
 * reference's seeding (spec.h:223-288), grid rule (spec.h:201-208), reaction
 * and IMEX arithmetic (spec.h:146-169, 394-408) so the tests can check the
 * oracle's restatement of them against the reference itself.
 */
#include "spec.h"

extern "C" {

void shtb_ref_grid_for_lmax(int lmax, int pdeg, int *nlat, int *nphi) {
  shtb_grid_for_lmax(lmax, pdeg, nlat, nphi);
}

long shtb_ref_nlm(int lmax, int mmax) { return shtb_nlm_calc(lmax, mmax); }

void shtb_ref_seeded_noise(long npts, double amp, unsigned seed, float *out) {
  shtb_seeded_noise(npts, amp, (uint32_t)seed, out);
}

void shtb_ref_seeded_spectrum(int lmax, int mmax, unsigned seed, float *qlm) {
  shtb_seeded_spectrum(lmax, mmax, (uint32_t)seed, qlm);
}

/* model: 0 schnakenberg, 1 brusselator, 2 allen-cahn (spec.h:43) with the
 * model's own default parameters (spec.h:59-67), evaluated at float. */
void shtb_ref_react_f32(int model, const float *u, const float *v, long n, float *r1,
                        float *r2) {
  const shtb_model_def *m = shtb_model_by_id(model);
  shtb_params p;
  shtb_default_params(m, &p);
  shtb_step_const<float> c = shtb_make_step_const<float>(m, &p);
  for (long i = 0; i < n; i++) {
    float a = 0, b = 0;
    shtb_react<float>(c, u[i], v ? v[i] : 0.0f, &a, &b);
    r1[i] = a;
    if (r2) r2[i] = b;
  }
}

void shtb_ref_react_f64(int model, const double *u, const double *v, long n, double *r1,
                        double *r2) {
  const shtb_model_def *m = shtb_model_by_id(model);
  shtb_params p;
  shtb_default_params(m, &p);
  shtb_step_const<double> c = shtb_make_step_const<double>(m, &p);
  for (long i = 0; i < n; i++) {
    double a = 0, b = 0;
    shtb_react<double>(c, u[i], v ? v[i] : 0.0, &a, &b);
    r1[i] = a;
    if (r2) r2[i] = b;
  }
}

/* One IMEX element update at float with the model's default parameters. */
float shtb_ref_imex_f32(int model, int k, float U, float R, float lam) {
  const shtb_model_def *m = shtb_model_by_id(model);
  shtb_params p;
  shtb_default_params(m, &p);
  shtb_step_const<float> c = shtb_make_step_const<float>(m, &p);
  return shtb_imex<float>(c, k, U, R, lam);
}

void shtb_ref_default_params(int model, double *a, double *b, double *D1, double *D2,
                             double *dt, double *eps2) {
  const shtb_model_def *m = shtb_model_by_id(model);
  shtb_params p;
  shtb_default_params(m, &p);
  *a = (model == 1) ? p.A : p.a;
  *b = (model == 1) ? p.B : p.b;
  *D1 = p.D1;
  *D2 = p.D2;
  *dt = p.dt;
  *eps2 = p.eps2;
}

}  // extern "C"
