// ref_extras — the reference's own extra order parameters (src/parameter_order.cpp:129-245: Polarization,
// Splay_magnitude, Splay_divergence, Radial_order) and its local order parameter (lattice_order_parameter,
// :75-127) behind C entry points, compiled from the reference sources with the GSL shim. Test infrastructure
// only: tests/test_extras_pin.py pins oracle/extras.py, the checker of the device extras, to these functions.
#include <string.h>

#include "../include/parameter_order.h"
#include "../include/parameters.h"
#include "../include/potential.h"

static Parameters lattice_params(int nx, int ny, int nz, const int periodic[3]) {
  Parameters p;
  p.Nx = nx;
  p.Ny = ny;
  p.Nz = nz;
  p.XBound = periodic[0] ? Periodic_Boundary : Free_Boundary;
  p.YBound = periodic[1] ? Periodic_Boundary : Free_Boundary;
  p.ZBound = periodic[2] ? Periodic_Boundary : Free_Boundary;
  return p;
}

// out: P, dtheta, divn, Sr_sph, Pr_sph, Sr_cyl, Pr_cyl (each function once, as ExtraObservables::accumulate calls
// them for one measurement sweep).
extern "C" void mcr_extras(int nx, int ny, int nz, const int periodic[3], float *ni, int *pt, float *director,
                           double out[7]) {
  Parameters p = lattice_params(nx, ny, nz, periodic);
  out[0] = Polarization(ni, pt, director, p);
  out[1] = Splay_magnitude(ni, pt, p);
  out[2] = Splay_divergence(ni, pt, p);
  Radial_order(ni, pt, p, false, out[3], out[4]);
  Radial_order(ni, pt, p, true, out[5], out[6]);
}

extern "C" float mcr_local_order(int nx, int ny, int nz, const int periodic[3], float *ni, int *pt, int i, int j,
                                 int k) {
  Parameters p = lattice_params(nx, ny, nz, periodic);
  return lattice_order_parameter(ni, pt, i, j, k, p);
}
