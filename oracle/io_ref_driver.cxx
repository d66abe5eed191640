// Test oracle driver for the reference's file formats (test infrastructure,
// built by oracle/Makefile into oracle/_ref/io_ref; never linked by the
// product).  It runs the reference's own writers and readers, unmodified:
//
//   io_ref dat IN DIR OUT   bodies from IN (int64 n, then n x {x, y, z, q, pot,
//                           ax, ay, az} float64) are written by
//                           Dataset::writeSources / writeTargets as
//                           DIR/source0000.dat and DIR/target0000.dat
//                           (exafmm include/dataset.h:313-372); both files are
//                           then read back twice in a row by readSources /
//                           readTargets (the second read continues at the
//                           stream position the first left), and OUT gets the
//                           values read: 2 x n x 8 float64
//   io_ref csv FILE v...    one RankCSV row with the example's main.csv
//                           columns (ex/tapas_exafmm.cxx:651-677, COUNT
//                           build): total upward traverse downward tree as
//                           doubles, numP2P numM2L as unsigned 64-bit, dumped
//                           by tapas::util::RankCSV (cpp/include/tapas/util.h)
#include <mpi.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "dataset.h"
#include "tapas/util.h"

int main(int argc, char **argv) {
  MPI_Init(&argc, &argv);
  if (argc >= 5 && std::string(argv[1]) == "dat") {
    FILE *f = fopen(argv[2], "rb");
    if (!f) return 1;
    int64_t n = 0;
    if (fread(&n, 8, 1, f) != 1) return 1;
    std::vector<double> v((size_t)n * 8);
    if (fread(v.data(), 8, v.size(), f) != v.size()) return 1;
    fclose(f);
    Bodies bodies((size_t)n);
    for (int64_t i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) bodies[i].X[d] = v[8 * i + d];
      bodies[i].SRC = v[8 * i + 3];
      for (int d = 0; d < 4; d++) bodies[i].TRG[d] = v[8 * i + 4 + d];
    }
    if (chdir(argv[3]) != 0) return 1;
    Dataset writer;
    writer.writeSources(bodies, 0);
    writer.writeTargets(bodies, 0);
    // read back: the halves of the file in two calls of n/2 and n - n/2 bodies
    Dataset reader;
    Bodies a((size_t)(n / 2)), b((size_t)(n - n / 2));
    reader.readSources(a, 0);
    reader.readSources(b, 0);
    Dataset treader;
    treader.readTargets(a, 0);
    treader.readTargets(b, 0);
    FILE *o = fopen(argv[4], "wb");
    if (!o) return 1;
    for (auto *part : {&a, &b})
      for (auto &body : *part) {
        double r[8] = {body.X[0], body.X[1], body.X[2], body.SRC,
                       body.TRG[0], body.TRG[1], body.TRG[2], body.TRG[3]};
        fwrite(r, 8, 8, o);
      }
    fclose(o);
  } else if (argc >= 10 && std::string(argv[1]) == "csv") {
    tapas::util::RankCSV csv{"total", "upward", "traverse", "downward", "tree", "numP2P",
                             "numM2L"};
    csv.At("total") = atof(argv[3]);
    csv.At("upward") = atof(argv[4]);
    csv.At("traverse") = atof(argv[5]);
    csv.At("downward") = atof(argv[6]);
    csv.At("tree") = atof(argv[7]);
    csv.At("numP2P") = (unsigned long)strtoull(argv[8], nullptr, 10);
    csv.At("numM2L") = (unsigned long)strtoull(argv[9], nullptr, 10);
    csv.Dump(std::string(argv[2]));
  } else {
    fprintf(stderr, "usage: %s dat IN DIR OUT | csv FILE total upward traverse downward tree "
                    "numP2P numM2L\n", argv[0]);
    return 2;
  }
  MPI_Finalize();
  return 0;
}
