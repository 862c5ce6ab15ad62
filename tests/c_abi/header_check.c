/* A plain C99 caller of include/turing_sht.h: compiled with -std=c99
 * -pedantic -Werror and linked against libturing_sht.so by
 * tests/test_c_header.py.  It calls only entry points that need no GPU
 * (layout algebra, seeding) plus ts_ctx_create, whose status it prints, so
 * it runs on a host without a GPU.  Exit status 0 when every check holds. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "turing_sht.h"

static int failures = 0;

#define CHECK(cond)                                      \
  do {                                                   \
    if (!(cond)) {                                       \
      fprintf(stderr, "check failed: %s\n", #cond);      \
      failures++;                                        \
    }                                                    \
  } while (0)

int main(void) {
  char msg[256];
  int nlat = 0, nphi = 0;
  float q[2 * 136];
  float noise[64];
  long i;
  ts_ctx ctx = NULL;
  int rc;

  CHECK(ts_nlm_calc(255, 255) == 32896L);
  CHECK(ts_nlm_calc(63, 63) == 2080L);
  CHECK(ts_lm_index(31, 31, 31) == ts_nlm_calc(31, 31) - 1);
  ts_grid_for_lmax(63, 3, &nlat, &nphi);
  CHECK(nlat == 128 && nphi == 256);
  CHECK(ts_validate_config(31, 31, 32, 64, msg, sizeof msg) == TS_OK);
  CHECK(ts_validate_config(31, 31, 32, 62, msg, sizeof msg) == TS_ERR_INVALID);
  CHECK(strstr(msg, "nphi must be") != NULL);

  ts_seeded_spectrum(15, 15, 1u, q);
  for (i = 0; i < 2 * 136; i++) CHECK(q[i] >= -1.0f && q[i] < 1.0f);
  for (i = 0; i <= 15; i++) CHECK(q[2 * i + 1] == 0.0f); /* m = 0 imaginary parts */
  ts_seeded_noise(64, 1e-2, 3u, noise);
  for (i = 0; i < 64; i++) CHECK(fabsf(noise[i]) < 1.0f);

  rc = ts_ctx_create(0, &ctx);
  printf("ts_ctx_create: %d (%s)\n", rc, rc == TS_OK ? "ok" : ts_last_error(NULL));
  if (rc == TS_OK) {
    ts_plan plan = NULL;
    CHECK(ts_sht_plan_create(ctx, 31, 31, 32, 64, TS_PREC_FP32, &plan) == TS_OK);
    if (plan) CHECK(ts_sht_plan_destroy(plan) == TS_OK);
    CHECK(ts_ctx_destroy(ctx) == TS_OK);
  } else {
    CHECK(rc == TS_ERR_CUDA || rc == TS_ERR_INVALID);
  }
  CHECK(ts_sht_synth_dev(NULL, NULL, NULL, 1, NULL) == TS_ERR_INVALID);
  printf("%s\n", failures ? "FAILED" : "ok");
  return failures ? 1 : 0;
}
