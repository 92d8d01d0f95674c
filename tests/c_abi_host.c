/* A plain C host of the library's host-only entry points (no device needed): the header compiles
 * as C, the quickhull of a cube with its centre, the error path of too few points, and the packing
 * of a scene's files (scene.json, scene.bin given on the command line) to the reference's packed
 * form. Prints one line per check; tests/test_c_abi_cpu.py builds and runs it. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "steel_b200.h"

static char* slurp(const char* path, uint64_t* len) {
  FILE* f = fopen(path, "rb");
  if (!f) return NULL;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  char* buf = (char*)malloc((size_t)n + 1);
  if (buf && fread(buf, 1, (size_t)n, f) != (size_t)n) { free(buf); buf = NULL; }
  if (buf) buf[n] = 0;
  fclose(f);
  *len = (uint64_t)n;
  return buf;
}

int main(int argc, char** argv) {
  /* A unit cube's corners and its centre: 8 vertices, 6 square faces on the planes |x|, |y|, |z| = 1. */
  double pts[9 * 3];
  int k = 0;
  for (int x = -1; x <= 1; x += 2)
    for (int y = -1; y <= 1; y += 2)
      for (int z = -1; z <= 1; z += 2) { pts[k++] = x; pts[k++] = y; pts[k++] = z; }
  pts[k++] = 0.0; pts[k++] = 0.0; pts[k++] = 0.0;
  double verts[27], planes[72];
  uint32_t start[19], fv[54], nv = 0, nf = 0;
  if (steel_convex_hull(pts, 9, verts, planes, start, fv, &nv, &nf) != STEEL_OK) {
    printf("hull failed: %s\n", steel_last_error());
    return 1;
  }
  int square = 1;
  for (uint32_t f = 0; f < nf; f++) {
    const double* p = planes + 4 * f;
    square = square && start[f + 1] - start[f] == 4 && fabs(p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - 1.0) < 1e-12 &&
             fabs(p[3] - 1.0) < 1e-12;
  }
  printf("hull %u %u %s\n", nv, nf, square ? "square" : "other");
  int rc = steel_convex_hull(pts, 3, verts, planes, start, fv, &nv, &nf);
  printf("few %d %s\n", rc, steel_last_error());
  if (argc >= 3) {
    uint64_t jl = 0, bl = 0;
    char* js = slurp(argv[1], &jl);
    char* bn = slurp(argv[2], &bl);
    steel_packed* pk = NULL;
    steel_scene_desc d;
    if (!js || !bn || steel_pack(js, jl, bn, bl, NULL, &pk) != STEEL_OK || steel_packed_desc(pk, &d) != STEEL_OK) {
      printf("pack failed: %s\n", steel_last_error());
      return 1;
    }
    printf("pack %llu %llu %llu\n", (unsigned long long)d.statF_floats, (unsigned long long)d.statU_words,
           (unsigned long long)d.art_floats);
    steel_packed_free(pk);
    free(js);
    free(bn);
  }
  steel_ctx* ctx = NULL;
  rc = steel_ctx_create(0, &ctx);
  printf("device %d\n", rc);
  if (rc == STEEL_OK) steel_ctx_destroy(ctx);
  return 0;
}
