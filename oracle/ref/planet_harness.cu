// planet_harness.cu -- runs the reference's own planet host code for one
// compiled-in disk (TEST INFRASTRUCTURE: golden vectors for the planet's
// orbit arithmetic, never part of the product).  No CUDA call is made; it
// runs without a GPU.
//
// usage: planet_ref <forces.bin> <rows.bin> <nsteps> <dt>
//   forces.bin: 2*nsteps doubles, the disk's (fx, fy) of each step.
//   rows.bin:   (nsteps + 1) rows of 12 doubles:
//     m x y vx vy fx fy rs (struct body), FrRot, get_ecc, get_E, set_M_p(t)
//   row 0 is init_planet (planet.cu:36-52) at t = 0; row n+1 follows step n:
//   fx, fy from the file, kick_drift_kick (planet.cu:67-93) with kick over
//   dt/2, drift over dt, kick over dt/2, at t = (n+1) dt.
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include <math.h>

#include "variable_types.h"
#include "global.h"
#include "planet.h"

using namespace std;

sdp set_M_p(sdp t);   // planet.cu:28-34 (not declared in planet.h)

static void record(vector<double> &rows, body &pl, sdp FrRot, sdp t) {
  const double r[12] = {pl.m, pl.x, pl.y, pl.vx, pl.vy, pl.fx, pl.fy, pl.rs, FrRot,
                        get_ecc(pl, FrRot), get_E(pl, FrRot), set_M_p(t)};
  rows.insert(rows.end(), r, r + 12);
}

int main(int argc, char **argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s <forces.bin> <rows.bin> <nsteps> <dt>\n", argv[0]);
    return 2;
  }
  const int nsteps = atoi(argv[3]);
  const double dt = strtod(argv[4], nullptr);
  vector<double> F(2 * (size_t)nsteps);
  FILE *f = fopen(argv[1], "rb");
  if (!f || fread(F.data(), sizeof(double), F.size(), f) != F.size()) return 3;
  fclose(f);
  body pl;
  sdp FrRot = 0.0;
  init_planet(pl, FrRot);
  pl.fx = 0.0;
  pl.fy = 0.0;
  vector<double> rows;
  record(rows, pl, FrRot, 0.0);
  for (int n = 0; n < nsteps; n++) {
    pl.fx = F[2 * n];
    pl.fy = F[2 * n + 1];
    kick_drift_kick(pl, FrRot, nullptr, 0.0, 0.5 * dt, true);
    kick_drift_kick(pl, FrRot, nullptr, 0.0, dt, false);
    kick_drift_kick(pl, FrRot, nullptr, 0.0, 0.5 * dt, true);
    record(rows, pl, FrRot, (n + 1) * dt);
  }
  f = fopen(argv[2], "wb");
  if (!f || fwrite(rows.data(), sizeof(double), rows.size(), f) != rows.size()) return 4;
  fclose(f);
  printf("{\"rows\": %d}\n", nsteps + 1);
  return 0;
}
