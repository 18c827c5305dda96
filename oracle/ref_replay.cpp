// ref_replay — drives the reference's own CPU Monte Carlo code (compiled from the reference sources with the
// GSL shim) with a replayed random stream, and dumps the state before every sweep. Test infrastructure only.
//
//   mclics_ref_replay <input_file> <n_sweeps> <seed64> <out.bin>
//
// The setup follows main.cpp:86-107 and simulator.cpp:32-126 step by step, calling the reference's functions,
// except that the director and point-type arrays stay in this program's hands. Each sweep t consumes the
// Philox uniforms of (seed64, sweep t) in the reference CPU's own call order (mc_oracle's mco_ref8_stream),
// with OMP_NUM_THREADS forced to 1 (evolve.cpp:106-201).
//
// out.bin (little endian): "MCLR" int32 version=1, int32 Nx, Ny, Nz, n_sweeps, int32 potential, flipMove,
// n_surfaces, int32 periodic x, y, z; float A, B1, C, lambda, mu, nu, rho, sigma, elecX, elecY, elecZ, elecA, elecP, elecE, T;
// per surface: int32 type, float W, theta, phi; int32 pt[Nt]; float ns[3 Nt]; then per sweep t:
// float ang_var_before, float ni_before[3 Nt], int32 n_draws, float E_after (energy_calculator), float
// ang_var_after; finally float ni_final[3 Nt].
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <map>
#include <string>
#include <vector>

#include "../include/define.h"
#include "../include/evolve.h"
#include "../include/geometry.h"
#include "../include/ic.h"
#include "../include/io.h"
#include "../include/parameters.h"
#include "../include/potential.h"
#include "gsl/gsl_rng.h"
#include "mc_oracle.h"

// EvolveN with its protected members reachable (no behaviour change).
struct ReplayEvolve : public EvolveN {
  ReplayEvolve(float *ni, int *pt, Parameters *p) : EvolveN(ni, pt, p) {}
};

static int anch_code(const std::string &s) {
  const char *n = s.c_str();
  if (!strcasecmp(n, "homeotropic")) return MCO_ANCH_HOMEOTROPIC;
  if (!strcasecmp(n, "rp")) return MCO_ANCH_RP;
  if (!strcasecmp(n, "rp_tangent")) return MCO_ANCH_RP_TANGENT;
  if (!strcasecmp(n, "fg")) return MCO_ANCH_FG;
  if (!strcasecmp(n, "homeotropic_ghrl")) return MCO_ANCH_HOMEOTROPIC_GHRL;
  if (!strcasecmp(n, "rp_ghrl")) return MCO_ANCH_RP_GHRL;
  if (!strcasecmp(n, "fg_ghrl")) return MCO_ANCH_FG_GHRL;
  return -1;
}

int main(int argc, char **argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s input n_sweeps seed64 out.bin\n", argv[0]);
    return 2;
  }
  omp_set_num_threads(1);
  const int n_sweeps = atoi(argv[2]);
  const unsigned long long seed64 = strtoull(argv[3], 0, 0);

  // main.cpp:86-107
  Parameters params = read_input_file(argv[1]);
  params.flipMove = (strcasecmp(params.potential, "pear") == 0 || params.elecP != 0) ? 1 : 0;
  if (params.MCQ < 0) params.MCQ = params.MCT;
  if (params.radial[0] == '\0') strcpy(params.radial, strcasecmp(params.geometry, "sphere") == 0 ? "sphere" : "none");
  if (params.elecA != 0 || params.elecP != 0) {
    float norm = sqrtf(params.elecX * params.elecX + params.elecY * params.elecY + params.elecZ * params.elecZ);
    params.elecX /= norm;
    params.elecY /= norm;
    params.elecZ /= norm;
  }
  validate_parameters(params);

  // simulator.cpp:32-126, keeping ni and pt here
  const int Nx = params.Nx, Ny = params.Ny, Nz = params.Nz, Nt = Nx * Ny * Nz;
  float *ni = (float *)calloc(3 * Nt, sizeof(float));
  int *pt = (int *)calloc(3 * Nt, sizeof(int));
  ReplayEvolve *ev = new ReplayEvolve(ni, pt, &params);
  if (strcasecmp(params.geometry, "bulk") == 0)
    ev->geometry = new Bulk_Geometry(pt, &params);
  else if (strcasecmp(params.geometry, "slab") == 0)
    ev->geometry = new Slab_Geometry(pt, &params);
  else if (strcasecmp(params.geometry, "sphere") == 0)
    ev->geometry = new Sphere_Geometry(pt, &params);
  else if (strcasecmp(params.geometry, "custom") == 0)
    ev->geometry = new Custom_Geometry(pt, &params);
  else {
    fprintf(stderr, "unknown geometry\n");
    return 2;
  }
  params.XBound = strcasecmp(params.XBoundtype, "periodic") == 0 ? &Periodic_Boundary : &Free_Boundary;
  params.YBound = strcasecmp(params.YBoundtype, "periodic") == 0 ? &Periodic_Boundary : &Free_Boundary;
  params.ZBound = strcasecmp(params.ZBoundtype, "periodic") == 0 ? &Periodic_Boundary : &Free_Boundary;
  check_checkerboard(params);
  ev->geometry->Boundary_Init(&params);
  apply_Initial_Conditions(ni, pt, params);
  int pot_code = MCO_POT_LL;
  if (strcasecmp(params.potential, "ll") * strcasecmp(params.potential, "lebwohl-lasher") == 0) {
    ev->geometry->bulk_potential = &Bulk_Energy_Lebwohl_Lasher;
  } else if (strcasecmp(params.potential, "ghrl") * strcasecmp(params.potential, "gruhn-hess") == 0) {
    ev->geometry->bulk_potential = &Bulk_Energy_GHRL;
    setGHRL(params);
    pot_code = MCO_POT_GHRL;
  } else {
    ev->geometry->bulk_potential = &Bulk_Energy_Selinger_Pear;
    pot_code = MCO_POT_PEAR;
  }
  params.T = params.Ti;

  mco_model m;
  memset(&m, 0, sizeof(m));
  m.potential = pot_code;
  m.flip_move = params.flipMove;
  mco_lattice L;
  memset(&L, 0, sizeof(L));
  L.nx = Nx;
  L.ny = Ny;
  L.nz = Nz;
  L.pt = pt;

  FILE *f = fopen(argv[4], "wb");
  if (!f) {
    perror(argv[4]);
    return 2;
  }
  auto wi = [&](int v) { fwrite(&v, 4, 1, f); };
  auto wf = [&](float v) { fwrite(&v, 4, 1, f); };
  fwrite("MCLR", 1, 4, f);
  wi(1);
  wi(Nx);
  wi(Ny);
  wi(Nz);
  wi(n_sweeps);
  wi(pot_code);
  wi(params.flipMove);
  const int nS = ev->geometry->nSurfaces;
  wi(nS);
  wi(strcasecmp(params.XBoundtype, "periodic") == 0);
  wi(strcasecmp(params.YBoundtype, "periodic") == 0);
  wi(strcasecmp(params.ZBoundtype, "periodic") == 0);
  float hdr[] = {params.A, params.B1, params.C, params.ghrl_lambda, params.ghrl_mu, params.ghrl_nu, params.ghrl_rho,
                 params.ghrl_sigma, params.elecX, params.elecY, params.elecZ, params.elecA, params.elecP, params.elecE,
                 params.T};
  fwrite(hdr, 4, sizeof(hdr) / 4, f);
  for (int s = 0; s < nS; s++) {
    wi(anch_code(params.anchoring_type.at(s)));
    wf(params.W.count(s) ? params.W[s] : 0.f);
    wf(params.theta_s.count(s) ? params.theta_s[s] : 0.f);
    wf(params.phi_s.count(s) ? params.phi_s[s] : 0.f);
  }
  fwrite(pt, 4, Nt, f);
  fwrite(ev->geometry->ns, 4, 3 * Nt, f);

  gsl_rng *r = gsl_rng_alloc(gsl_rng_ranlxs0);
  gsl_rng *rr[1] = {r};
  float ang_var = 0.5f;
  std::vector<double> stream((size_t)Nt * 4 + 16);
  for (int t = 0; t < n_sweeps; t++) {
    wf(ang_var);
    fwrite(ni, 4, 3 * Nt, f);
    int64_t n = mco_ref8_stream(&m, &L, seed64, (uint64_t)t, stream.data(), (int64_t)stream.size());
    gslshim_set_replay(stream.data(), (size_t)n);
    ev->Monte_Carlo_Step(ang_var, rr);
    size_t used = gslshim_replay_consumed();
    gslshim_clear_replay();
    if ((int64_t)used != n) {
      fprintf(stderr, "replay: sweep %d consumed %zu of %lld draws\n", t, used, (long long)n);
      return 3;
    }
    wi((int)n);
    wf(ev->energy_calculator());
    wf(ang_var);
  }
  fwrite(ni, 4, 3 * Nt, f);
  fclose(f);
  return 0;
}
