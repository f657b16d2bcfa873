// grid_harness.cu -- runs the reference's own host grid generator (grid() of
// src/shared/grid.cu, compiled into the reference's src/shared/global.cu)
// for a list of grid types and ranges, and writes the face, centre and width
// arrays (TEST INFRASTRUCTURE: golden vectors for the grid generator, never
// part of the product).
//
// usage: grid_ref <out.bin> lg,nzones,lo,hi [lg,nzones,lo,hi ...]
// out.bin: per case nzones doubles of xa, then xc, then dx.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>
using namespace std;   // the reference's headers name string unqualified

#include "variable_types.h"
#include "global.h"

void grid(int start, int nzones, sdp xmin, sdp xmax, sdp *xa, sdp *xc, sdp *dx, int lg);

int main(int argc, char **argv) {
  if (argc < 3) { fprintf(stderr, "usage: %s out.bin lg,n,lo,hi ...\n", argv[0]); return 2; }
  FILE *f = fopen(argv[1], "wb");
  if (!f) return 3;
  for (int a = 2; a < argc; a++) {
    int lg = 0, n = 0;
    double lo = 0.0, hi = 0.0;
    if (sscanf(argv[a], "%d,%d,%la,%la", &lg, &n, &lo, &hi) != 4 || n < 2) { fclose(f); return 4; }
    std::vector<double> xa(n, 0.0), xc(n, 0.0), dx(n, 0.0);
    grid(0, n, lo, hi, xa.data(), xc.data(), dx.data(), lg);
    fwrite(xa.data(), sizeof(double), n, f);
    fwrite(xc.data(), sizeof(double), n, f);
    fwrite(dx.data(), sizeof(double), n, f);
  }
  fclose(f);
  return 0;
}
