// pg_host.h -- host-side set-up shared by the run object (pg_run.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/penguin_b200.h"

namespace pg {

extern const double kTwoPi, kPi, kHalfPi, kThird, kEarthMass;

// Disk profile of disk_profile.cu evaluated with the run's parameters.
struct Profile {
  pg_params P;
  double rho(double r) const;
  double rho(double r, double z) const;
  double cs2(double r) const;
  double h(double r) const;
  double pres(double r) const;
  double pres(double r, double z) const;
  double dP_dr(double r) const;
  double dP_s(double r, double pol) const;
  double verfac(double r, double z) const;
  double nu(double r) const;
  double viscous_vr(double r) const;
  double vol(double xa, double dx, int axis) const;
};

struct SymDisk { double r, p, u, v, w; };

// A fixed boundary ring: geometry plus its phi-uniform state.
struct GhostRing {
  double x, dx, xvol, xc, z, dz, zvol, zc;
  double r, p, u, v, w, rot_v;
};

struct Geometry {
  std::vector<double> zxa, zxc, zdx, xvol;
  std::vector<double> zya, zyc, zdy, yvol;
  std::vector<double> zza, zzc, zdz, zvol;
};

// Byte view of one hydr_ring record.  f(0..4) = r,p,u,v,w; scal(0..3) =
// x,dx,xvol,xc; col(0..3) = y,dy,yvol,yc; zs(0..3) = z,dz,zvol,zc;
// ik(0..1) = i,k; rot(0..1) = rot_v,res_v; rj(0..1) = rot_j,inc_j.
struct RingView {
  unsigned char *base;
  int n;
  RingView(unsigned char *b, int jmax);
  double *f(int field) const;
  double *scal(int which) const;
  double *col(int which) const;
  double *zs(int which) const;
  int *ik(int which) const;
  double *rot(int which) const;
  int *rj(int which) const;
};

size_t ring_bytes(int jmax);
void default_params(pg_params *p);
int config_params(int which, pg_params *p);
int check_params(const pg_params *p, std::string &why);
int build_ic(const pg_params *p, void *buf, size_t bytes, std::string &why);
double ic_uniform(uint64_t seed, uint64_t idx);
void build_val(const Profile &pf, const std::vector<double> &zxc, const std::vector<double> &zzc,
               std::vector<SymDisk> &val);
GhostRing make_ghost(const Profile &pf, double x, double dx, double xc, double z, double dz,
                     double zc, int theta_layer);
void boundary_rings(const Profile &pf, const Geometry &g, std::vector<GhostRing> &lft,
                    std::vector<GhostRing> &rgh, std::vector<GhostRing> &udr, std::vector<GhostRing> &top);
int params_geometry(const pg_params &P, Geometry &g);
// pow(x, y) in the form the reference's compiler gives a constant exponent
double cpow_c(double x, double y);
int read_geometry(const pg_params &P, const unsigned char *b, Geometry &g, std::string &why);
std::string label(const pg_params &P);

}  // namespace pg
