// post_harness.cpp -- runs the reference's own read/ post-processing on a
// dump, on the host (TEST INFRASTRUCTURE: golden values for the device
// post-processing, never part of the product).
//
// The reference's offline tools (read/post.cu) need MathGL for their plots,
// but the two routines restated on the device do not: get_torque
// (read/transform.cpp:386-420) and write_har_file (read/p_output.cpp:35-55).
// This driver declares the globals post.cu declares and #includes the
// reference's read/rk_high.cpp, transform.cpp, p_init.cpp and p_output.cpp
// where they lie, against a per-workload copy of include/post_global.h
// (grid sizes and M_p patched by oracle/ref/gen_headers.py).  It loads a
// dump with the reference's own copy_grid and update_grid (p_init.cpp:79-133,
// the de-rotation), then prints get_torque() and, for each requested m, the
// an/bn columns write_har_file echoes to stdout (at 17 digits).
//
// usage: post_ref <dump> <m1,m2,...>
#include <unistd.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#define __host__
#define __device__
struct double2 { double x, y; };
struct dim3 { unsigned x, y, z; };
typedef void *cudaEvent_t;
typedef void *cudaStream_t;

#include "post_global.h"

// the globals of read/post.cu:16-48 (image sizes are used by the image
// conversion only, which this driver never calls)
const int imgDimx = 500;
const int imgDimy = 500;
const int imgDimz = 1;
vector<vector<vector<sdp> > > zro, zpr, zux, zuy, zuz;
int nDev;
sdp gam, sc_h, simtime, tmovie;
string mainp, label;
int grspx, grspy, grspz;
sdp xmin, xmax, ymin, ymax, zmin, zmax;
sdp *zxa, *zxc, *zdx, *zya, *zyc, *zdy, *zza, *zzc, *zdz;

// grid() is declared by post_global.h and used only by init_grid, which this
// driver never calls (the dump carries the grid); defined in src/shared
// with the reference's configuration types, it is stubbed here
void grid(int, int, sdp, sdp, sdp *, sdp *, sdp *, int) { std::abort(); }
// the same for the interactive pause of the streamline tracer
void wait_f_r() { std::abort(); }

#include "read/rk_high.cpp"
#include "read/transform.cpp"
#include "read/p_init.cpp"
#include "read/p_output.cpp"

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <dump> <m1,m2,...>\n", argv[0]);
    return 2;
  }
  nDev = 1;
  GPU_plan set[1];
  set[0].N_ring = imax * kmax;
  set[0].h_rings = new hydr_ring[imax * kmax];
  std::ifstream f(argv[1], std::ios::in | std::ios::binary);
  f.read((char *)set[0].h_rings, (std::streamsize)sizeof(hydr_ring) * imax * kmax);
  if (!f) { std::fprintf(stderr, "short read of %s\n", argv[1]); return 3; }
  zxa = new sdp[imax]; zxc = new sdp[imax]; zdx = new sdp[imax];
  zya = new sdp[jmax]; zyc = new sdp[jmax]; zdy = new sdp[jmax];
  zza = new sdp[kmax]; zzc = new sdp[kmax]; zdz = new sdp[kmax];
  set_size_for_data();
  copy_grid(set);
  update_grid(set);
  std::printf("torque %a\n", get_torque());
  std::fflush(stdout);
  std::cout << std::setprecision(17);
  std::stringstream ms(argv[2]);
  std::string tok;
  while (std::getline(ms, tok, ',')) {
    std::cout << "harmonic " << tok << std::endl;
    write_har_file(std::atof(tok.c_str()), "/dev/null");
  }
  return 0;
}
