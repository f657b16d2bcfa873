// ic_harness.cu -- runs the reference's own initial set-up on the host:
// init_grid, init_den, init_speed, init_cells and init_bound (init.cpp:3-543)
// for one compiled-in disk, then writes the initial dump (save_cells,
// output.cu:48-55) and the fixed boundary rings lft, rgh, udr, top as raw
// hydr_ring records (TEST INFRASTRUCTURE: golden vectors for the initial
// state and the boundary rings, never part of the product).  No CUDA call is
// made; it runs without a GPU.
//
// usage: ic_ref <outdir>   -> <outdir>/ic_ref.bin, <outdir>/boundary.bin
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <math.h>

#include "variable_types.h"
#include "global.h"
#include "disk_profile.h"
#include "output.h"

using namespace std;

sdp *zxa, *zxc, *zdx, *zya, *zyc, *zdy, *zza, *zzc, *zdz;

#include "init.cpp"

int main(int argc, char **argv) {
  if (argc < 2) { fprintf(stderr, "usage: %s <outdir>\n", argv[0]); return 2; }
  string out = argv[1];
  zxa = new sdp[imax]; zxc = new sdp[imax]; zdx = new sdp[imax];
  zya = new sdp[jmax]; zyc = new sdp[jmax]; zdy = new sdp[jmax];
  zza = new sdp[kmax]; zzc = new sdp[kmax]; zdz = new sdp[kmax];
  init_grid();
  SymDisk *val = new SymDisk[imax * kmax];
  init_den(val);
  init_speed(val);
  GPU_plan *set = new GPU_plan[1];
  set[0].N_ring = imax * kmax;
  set[0].memsize = set[0].N_ring * sizeof(hydr_ring);
  set[0].istart = 0; set[0].iblk = imax;
  set[0].kstart = 0; set[0].kblk = kmax;
  set[0].h_rings = (hydr_ring *)calloc(set[0].N_ring, sizeof(hydr_ring));
  init_cells(set, val);
  ofstream of((out + "/ic_ref.bin").c_str(), ios::out | ios::binary);
  save_cells(of, set);
  of.close();
  // zeroed rings, as the run's harness allocates them (res_v, inc_j = 0)
  hydr_ring *lft = (hydr_ring *)calloc(n_pad * kmax, sizeof(hydr_ring));
  hydr_ring *rgh = (hydr_ring *)calloc(n_pad * kmax, sizeof(hydr_ring));
  hydr_ring *udr = (hydr_ring *)calloc(n_pad * imax, sizeof(hydr_ring));
  hydr_ring *top = (hydr_ring *)calloc(n_pad * imax, sizeof(hydr_ring));
  init_bound(lft, rgh, udr, top);
  FILE *f = fopen((out + "/boundary.bin").c_str(), "wb");
  if (!f) return 3;
  fwrite(lft, sizeof(hydr_ring), n_pad * kmax, f);
  fwrite(rgh, sizeof(hydr_ring), n_pad * kmax, f);
  fwrite(udr, sizeof(hydr_ring), n_pad * imax, f);
  fwrite(top, sizeof(hydr_ring), n_pad * imax, f);
  fclose(f);
  printf("{\"rings\": %d, \"ring_bytes\": %zu}\n", imax * kmax, sizeof(hydr_ring));
  return 0;
}
