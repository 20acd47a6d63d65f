/* A C11 caller of the library's host-only entry points, compiled and run by
 * tests/test_c_caller.py: the header is plain C, and the coefficient tables,
 * LU factors, exchange plans and record files work without a GPU or Python.
 * Prints one "name value" line per check and "ok" at the end. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "canard_gpu.h"

static int fail(const char* what, int rc) {
  printf("FAIL %s rc=%d\n", what, rc);
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 2) return fail("usage: host_abi DIR", 0);
  double coef[150];
  int rc = canard_coeffs(0.85, 0.85, coef);
  if (rc != CANARD_OK) return fail("canard_coeffs", rc);
  printf("coeffs0 %.17g\n", coef[0]);
  if (canard_coeffs(0.85, -1.0, NULL) != CANARD_ERR_ARG) return fail("canard_coeffs bad argument", 0);

  enum { N = 33 };
  double xu[3 * N], xl[2 * N]; /* (n,3) and (n,2) */
  rc = canard_penta(0.85, 0.85, N, 0, 0, 0, xu, xl);
  if (rc != CANARD_OK) return fail("canard_penta", rc);
  printf("penta_xu0 %.17g\n", xu[0]);

  /* a periodic box of two ranks split along zeta (code 40 between them,
     45 at the box's ends), as cases.decompose writes it */
  canard_block_desc r[2];
  memset(r, 0, sizeof r);
  for (int b = 0; b < 2; ++b) {
    r[b].lxi = 16; r[b].let = 16; r[b].lze = 15 - b; /* 30 cells split in two */
    for (int d = 0; d < 2; ++d) {
      r[b].nbc[d][0] = r[b].nbc[d][1] = 45;
      r[b].mbcd[d][0] = r[b].mbcd[d][1] = b;
    }
  }
  r[0].nbc[2][0] = 45; r[0].mbcd[2][0] = 1; r[0].nbc[2][1] = 40; r[0].mbcd[2][1] = 1;
  r[1].nbc[2][0] = 40; r[1].mbcd[2][0] = 0; r[1].nbc[2][1] = 45; r[1].mbcd[2][1] = 0;
  const int32_t nbpc[3] = {1, 1, 2}, mbcd[6] = {0, 0, 0, 0, 0, 0}, sub[8] = {0, 0, 0, 0, 0, 0, 0, 1};
  int64_t n = 0;
  rc = canard_plan_export(2, r, 1, nbpc, mbcd, sub, 0, NULL, 0, &n);
  if (rc != CANARD_OK) return fail("canard_plan_export size", rc);
  int64_t* links = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  if (canard_plan_export(2, r, 1, nbpc, mbcd, sub, 0, links, n - 1, &n) != CANARD_ERR_ARG)
    return fail("canard_plan_export short buffer", 0);
  rc = canard_plan_export(2, r, 1, nbpc, mbcd, sub, 0, links, n, &n);
  if (rc != CANARD_OK) return fail("canard_plan_export", rc);
  int cross = 0;
  for (int64_t i = 0; i < n / 7; ++i) cross += links[7 * i] != links[7 * i + 3];
  printf("links %lld\ncross %d\n", (long long)(n / 7), cross);
  free(links);

  /* restart file round trip in the reference's record format */
  char path[4096];
  snprintf(path, sizeof path, "%s/restart_c.da", argv[1]);
  enum { P = 40 };
  double t6[6] = {12, 3, 0.25, 0.5, 0.75, 1.5}, q[5 * P], t6b[6], qb[5 * P];
  for (int i = 0; i < 5 * P; ++i) q[i] = 0.5 * i - 3.0;
  rc = canard_restart_write_file(path, t6, q, P);
  if (rc != CANARD_OK) return fail("canard_restart_write_file", rc);
  rc = canard_restart_read_file(path, t6b, qb, P);
  if (rc != CANARD_OK) return fail("canard_restart_read_file", rc);
  if (memcmp(q, qb, sizeof q) != 0 || t6b[5] != t6[5] || t6b[2] != t6[2]) return fail("restart round trip", 0);
  if (canard_restart_read_file(path, t6b, qb, P + 1) != CANARD_ERR_IO) return fail("restart size check", 0);
  printf("ok\n");
  return 0;
}
