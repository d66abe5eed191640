// Test oracle driver around the UNMODIFIED reference Barnes-Hut sample
// (sample/barnes-hut/bh.cc).  Its `main` is renamed; the sample's own calc()
// (bh.cc:228-245: Partition with ncrit = 1, Approximate, interact with
// theta = 0.5, EPS2 = 1e-6) runs on bodies read from a file.
//
// Test infrastructure: built by oracle/Makefile into oracle/_ref/.
//
// Usage:  bh_ref IN OUT
//   IN : int64 n, then n x {x, y, z, w} float64
//   OUT: int64 n, then per body in the sample's (Morton) order
//        {x, y, z, w} of the body and {x, y, z, w} of its result
#define main bh_reference_main
#include "bh.cc"
#undef main

#include <cstdio>
#include <vector>

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s IN OUT\n", argv[0]);
    return 2;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 1;
  int64_t n = 0;
  if (fread(&n, 8, 1, f) != 1) return 1;
  f4vec src((size_t)n);
  for (int64_t i = 0; i < n; i++) {
    double v[4];
    if (fread(v, 8, 4, f) != 4) return 1;
    src[(size_t)i].x = v[0];
    src[(size_t)i].y = v[1];
    src[(size_t)i].z = v[2];
    src[(size_t)i].w = v[3];
  }
  fclose(f);
  MPI_Init(&argc, &argv);
  f4vec out = calc(src);
  FILE *g = fopen(argv[2], "wb");
  if (!g) return 1;
  fwrite(&n, 8, 1, g);
  for (int64_t i = 0; i < n; i++) {
    const double v[8] = {src[i].x, src[i].y, src[i].z, src[i].w,
                         out[i].x, out[i].y, out[i].z, out[i].w};
    fwrite(v, 8, 8, g);
  }
  fclose(g);
  MPI_Finalize();
  return 0;
}
