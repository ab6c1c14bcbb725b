/* A plain C99 consumer of include/ladds_gpu.h: what a maintainer's C / cgo /
 * FFI binding sees.  Host-only entry points (no device needed): the ABI
 * version, a generated population written to a population file and read back,
 * and the CSV record writer.  Exit status 0 = all checks passed. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ladds_gpu.h"

#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      fprintf(stderr, "%s:%d: %s\n", __FILE__, __LINE__, #c); \
      return 1;                                               \
    }                                                         \
  } while (0)

typedef struct {
  double *f[9];
  uint64_t *id, *parent;
  int8_t *act;
} Pop;

static int popAlloc(Pop *p, size_t n) {
  for (int k = 0; k < 9; ++k) p->f[k] = (double *)calloc(n ? n : 1, sizeof(double));
  p->id = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
  p->parent = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
  p->act = (int8_t *)calloc(n ? n : 1, 1);
  return p->id && p->parent && p->act;
}

int main(int argc, char **argv) {
  const char *dir = argc > 1 ? argv[1] : ".";
  CHECK(ladds_gpu_abi_version() >= 2);

  const size_t n = 2000;
  Pop a, b;
  CHECK(popAlloc(&a, n) && popAlloc(&b, n));
  CHECK(ladds_population_generate(0, 42, n, a.f[0], a.f[1], a.f[2], a.f[3], a.f[4], a.f[5], a.f[6], a.f[7], a.f[8],
                                  a.id, a.parent, a.act) == LADDS_OK);
  char path[4096];
  snprintf(path, sizeof path, "%s/pop.bin", dir);
  CHECK(ladds_population_write(path, n, a.f[0], a.f[1], a.f[2], a.f[3], a.f[4], a.f[5], a.f[6], a.f[7], a.f[8], a.id,
                               a.parent, a.act) == LADDS_OK);
  size_t got = 0;
  CHECK(ladds_population_read(path, n - 1, &got, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                              NULL) == LADDS_ERR_CAPACITY);
  CHECK(got == n);
  CHECK(ladds_population_read(path, n, &got, b.f[0], b.f[1], b.f[2], b.f[3], b.f[4], b.f[5], b.f[6], b.f[7], b.f[8],
                              b.id, b.parent, b.act) == LADDS_OK);
  for (int k = 0; k < 9; ++k) CHECK(memcmp(a.f[k], b.f[k], n * sizeof(double)) == 0);
  CHECK(memcmp(a.id, b.id, n * sizeof(uint64_t)) == 0 && memcmp(a.act, b.act, n) == 0);

  ladds_pair recs[2];
  memset(recs, 0, sizeof recs);
  recs[0].step = 3;
  recs[0].idA = 1;
  recs[0].idB = 2;
  recs[0].dl2 = 0.25;
  recs[0].flags = LADDS_PAIR_COLLISION;
  recs[1] = recs[0];
  recs[1].idB = 5;
  recs[1].flags = LADDS_PAIR_EVASION;
  snprintf(path, sizeof path, "%s/conj.csv", dir);
  CHECK(ladds_records_write_csv(path, 0, recs, 2, LADDS_PAIR_COLLISION) == LADDS_OK);
  FILE *f = fopen(path, "r");
  CHECK(f != NULL);
  char line[256];
  int lines = 0;
  while (fgets(line, sizeof line, f)) ++lines;
  fclose(f);
  CHECK(lines == 2); /* header + the one collision */

  CHECK(ladds_gpu_create(NULL, NULL) == LADDS_ERR_INVALID_ARG);
  printf("abi_consumer: ok\n");
  return 0;
}
