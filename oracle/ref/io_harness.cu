// io_harness.cu -- runs the reference's own output naming and text writers on
// the host for one compiled-in disk (TEST INFRASTRUCTURE: golden text for the
// run label, the dump names, the para file and the time file's number
// format, never part of the product).  No CUDA call is made; it runs without
// a GPU.
//
// usage: io_ref <outdir> <mainp> v0 ... v10
//   <outdir>/label.txt   create_label() (output.cu:57-88)
//   <outdir>/frames.txt  the dump name of main.cu:124 for frames 0, 7, 42,
//                        1234 and 99999 (frame_num, global.cu), one per line
//   <outdir>/para.dat    write_para_file (output.cu:90-109) through
//                        open_output_file (output.cu:14-23)
//   <outdir>/time.dat    v0..v10 as one time-file row (v0, v1 only without a
//                        planet): a stream opened by append_output_file
//                        (output.cu:25-34), values separated by one space,
//                        the row ended by endl (main.cu:417-427)
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <math.h>

#include "variable_types.h"
#include "global.h"
#include "output.h"

using namespace std;

int main(int argc, char **argv) {
  if (argc != 14) {
    fprintf(stderr, "usage: %s <outdir> <mainp> v0 ... v10\n", argv[0]);
    return 2;
  }
  string out = argv[1];
  string mainp = argv[2];
  string label = create_label();
  {
    ofstream f((out + "/label.txt").c_str());
    f << label;
  }
  {
    ofstream f((out + "/frames.txt").c_str());
    const int frames[] = {0, 7, 42, 1234, 99999};
    for (int n : frames) f << mainp + "/binary/binary_" + label + "_" + frame_num(n) << "\n";
  }
  {
    ofstream pfile;
    open_output_file(pfile, out + "/para.dat");
    write_para_file(pfile, mainp, label);
  }
  {
    ofstream tfile;
    append_output_file(tfile, out + "/time.dat");
    // without a planet the row stops after the mass (main.cu:419-425)
#if plnt_flag > 0
    const int ncols = 11;
#else
    const int ncols = 2;
#endif
    for (int c = 0; c < ncols; c++) {
      if (c) tfile << " ";
      tfile << strtod(argv[3 + c], nullptr);
    }
    tfile << endl;
  }
  printf("{\"label\": \"%s\"}\n", label.c_str());
  return 0;
}
