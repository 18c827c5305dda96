// Drop-in bodies of the reference's GPU evolution classes on this library's engine.
//
// The reference selects its GPU modes in simulator.cpp (src/simulator.cpp:45-53) by constructing
// thermalEvolveNGPU, stepEvolveNGPU, quenchEvolveNGPU or electricEvolveNGPU with (float *ni, int *pt,
// Parameters *params) (include/evolve.cuh:22-67) and calling run(). This file defines those constructors,
// destructors and run() methods over the C ABI of include/mclics_b200.h, in place of the reference's
// src/evolve_{thermal,step,quench,electric}.cu, evolve.cu, geometry.cu, potential.cu, reduce.cu and stringGPU.cu.
// Linking it with the reference's own host sources (main.cpp, simulator.cpp with CUDA__ defined, io.cpp, ...) gives
// the reference program with this engine behind its *GPU modes; adapter/Makefile is the recipe.
//
// What stays the reference's: the input file, the set-up (geometry, anchorings, initial condition, GHRL
// coefficients), the scan points and snapshot names (include/sweep.h), the po.dat lines and the extra columns
// (ExtraObservables), the snapshot writer (print_n). What the engine does: the sweeps, the energy, the Q tensor and
// S of every measurement sweep (on the device, FP64 sums), ang_var adaptation. The director field comes back to the
// host only for snapshots, and every measurement sweep when the run has extra po.dat columns (pear or radial),
// which the reference computes on the host from the whole field.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <vector>

#include "../include/evolve.cuh"
#include "../include/io.h"
#include "../include/parameter_order.h"
#include "../include/sweep.h"
#include "mclics_b200.h"

namespace {

// The reference reports a failed CUDA call and exits with status 20; the engine's message says what failed.
void ok(int rc) {
  if (rc == MCL_OK) return;
  fprintf(stderr, "  [ERROR] mclics_b200: %s\n", mcl_last_error());
  exit(20);
}

int code_of(const std::string &name, const char *const *names, const int *codes, int n) {
  for (int i = 0; i < n; i++)
    if (!strcasecmp(name.c_str(), names[i])) return codes[i];
  return -1;
}

mcl_model model_of(const Parameters &p, const Geometry *g) {
  static const char *const pots[] = {"ll", "lebwohl-lasher", "ghrl", "gruhn-hess", "pear"};
  static const int pot_codes[] = {MCL_POT_LL, MCL_POT_LL, MCL_POT_GHRL, MCL_POT_GHRL, MCL_POT_PEAR};
  static const char *const anchs[] = {"homeotropic", "rp", "rp_tangent", "fg", "homeotropic_ghrl", "rp_ghrl", "fg_ghrl"};
  static const int anch_codes[] = {MCL_ANCH_HOMEOTROPIC, MCL_ANCH_RP,     MCL_ANCH_RP_TANGENT, MCL_ANCH_FG,
                                   MCL_ANCH_HOMEOTROPIC_GHRL, MCL_ANCH_RP_GHRL, MCL_ANCH_FG_GHRL};
  mcl_model m;
  memset(&m, 0, sizeof m);
  m.potential = code_of(p.potential, pots, pot_codes, 5);
  m.A = p.A;
  m.B1 = p.B1;
  m.C = p.C;
  m.ghrl_lambda = p.ghrl_lambda;  // set by setGHRL during the reference's set-up
  m.ghrl_mu = p.ghrl_mu;
  m.ghrl_nu = p.ghrl_nu;
  m.ghrl_rho = p.ghrl_rho;
  m.ghrl_sigma = p.ghrl_sigma;
  m.field_dir[0] = p.elecX;  // normalised by main
  m.field_dir[1] = p.elecY;
  m.field_dir[2] = p.elecZ;
  m.elecA = p.elecA;
  m.elecP = p.elecP;
  m.flip_move = p.flipMove;
  m.n_surfaces = g->nSurfaces;
  for (int s = 0; s < g->nSurfaces && s < MCL_MAX_SURFACES; s++) {  // the set-up checked that each is defined
    m.anch_type[s] = code_of(p.anchoring_type.at(s), anchs, anch_codes, 7);
    m.anch_W[s] = p.W.at(s);
    m.anch_theta[s] = p.theta_s.count(s) ? p.theta_s.at(s) : 0.f;
    m.anch_phi[s] = p.phi_s.count(s) ? p.phi_s.at(s) : 0.f;
  }
  return m;
}

// One lattice of the reference's set-up as an engine replica, its directors uploaded.
mcl_engine *engine_of(float *ni, int *pt, Parameters *p, Geometry *g) {
  mcl_replica r;
  memset(&r, 0, sizeof r);
  r.nx = p->Nx;
  r.ny = p->Ny;
  r.nz = p->Nz;
  r.geometry = !strcasecmp(p->geometry, "slab")     ? MCL_GEOM_SLAB
               : !strcasecmp(p->geometry, "sphere") ? MCL_GEOM_SPHERE
               : !strcasecmp(p->geometry, "custom") ? MCL_GEOM_CUSTOM
                                                    : MCL_GEOM_BULK;
  r.periodic[0] = !strcasecmp(p->XBoundtype, "periodic");
  r.periodic[1] = !strcasecmp(p->YBoundtype, "periodic");
  r.periodic[2] = r.geometry == MCL_GEOM_SLAB ? 0 : !strcasecmp(p->ZBoundtype, "periodic");
  r.T = p->Ti;
  r.elecE = 1.f;
  r.ang_var = 0.5f;  // once per run (src/evolve_thermal.cu:43)
  r.seed = (unsigned long long)(long long)p->seed;
  const mcl_model m = model_of(*p, g);
  mcl_engine *e = nullptr;
  ok(mcl_create(&m, &r, 1, MCL_SCHED_CHECKER2, &e));
  if (r.geometry == MCL_GEOM_SPHERE || r.geometry == MCL_GEOM_CUSTOM) ok(mcl_set_geometry(e, 0, pt, g->ns));
  ok(mcl_upload_directors(e, 0, ni));
  return e;
}

enum Mode { THERMAL, STEP, QUENCH, ELECTRIC };

// The loop of the four modes: scan points (temperatures, blocks or field values), MCT (and MCQ) sweeps before each,
// MCS measured sweeps, one po.dat line and one snapshot per point.
int run_mode(Mode mode, float *ni, int *pt, Parameters *p, Geometry *g) {
  mcl_engine *e = engine_of(ni, pt, p, g);
  ExtraObservables extra(p);
  const bool extras = !strcasecmp(p->potential, "pear") || !strcasecmp(p->radial, "sphere") ||
                      !strcasecmp(p->radial, "cylinder") || !strcasecmp(p->radial, "both");
  ok(mcl_reserve_series(e, p->MCS));
  FILE *po = fopen("po.dat", "a");
  if (!po) {
    perror("po.dat");
    exit(2);
  }
  const char *first = mode == THERMAL ? "T" : (mode == ELECTRIC ? "field" : "ii");
  fprintf(po, "%s S varS E varE", first);
  extra.write_header(po);
  fflush(po);
  const double step = mode == ELECTRIC ? p->elecdE : p->dT;
  const int snapS = snapshot_scale(step);
  if (mode == THERMAL && snapS != 100) printf("  Snapshot names: director_field_<int(%d T)>.csv (|dT| < 0.01)\n", snapS);
  if (mode == ELECTRIC) printf("  Snapshot names: director_field_<int(%d E)>.csv\n", snapS);
  const int points = mode == THERMAL    ? sweep_points(p->Ti, p->Tf, p->dT)
                     : mode == ELECTRIC ? sweep_points(p->elecEi, p->elecEf, p->elecdE)
                                        : p->fn;
  p->T = p->Ti;
  std::vector<mcl_observables> obs(p->MCS);
  char fname[1000];
  for (int it = 0; it < points; it++) {
    if (mode == THERMAL) p->T = sweep_value(p->Ti, p->Tf, p->dT, it, points);
    if (mode == ELECTRIC) p->elecE = sweep_value(p->elecEi, p->elecEf, p->elecdE, it, points);
    if (mode == QUENCH) p->T = p->Ti;
    ok(mcl_set_temperature(e, 0, p->T));
    ok(mcl_set_field(e, 0, p->elecE));
    ok(mcl_sweeps(e, p->MCT, 0));
    if (mode == QUENCH) {
      p->T = p->Tf;
      ok(mcl_set_temperature(e, 0, p->T));
      ok(mcl_sweeps(e, p->MCQ, 0));
    }
    extra.reset();
    ok(mcl_clear_series(e));
    if (extras) {  // the extra columns need the whole field after every measured sweep, as in the reference
      for (int s = 0; s < p->MCS; s++) {
        ok(mcl_sweeps(e, 1, 1));
        ok(mcl_read_series(e, 0, s, 1, &obs[s]));
        ok(mcl_download_directors(e, 0, ni));
        float d[3] = {(float)obs[s].director[0], (float)obs[s].director[1], (float)obs[s].director[2]};
        extra.accumulate(ni, pt, d);
      }
    } else {
      ok(mcl_sweeps(e, p->MCS, 1));
      ok(mcl_read_series(e, 0, 0, p->MCS, obs.data()));
    }
    double S1 = 0, S2 = 0, E = 0, E2 = 0;
    for (const mcl_observables &o : obs) {
      const float tE = (float)o.energy, tS = (float)o.S;  // the reference's float energy and eigenvalue
      E += tE;
      E2 += tE * tE;
      S1 += tS;
      S2 += tS * tS;
    }
    E /= p->MCS;
    E2 /= p->MCS;
    S1 /= p->MCS;
    S2 /= p->MCS;
    ok(mcl_download_directors(e, 0, ni));
    if (mode == THERMAL)
      sprintf(fname, "director_field_%ld.csv", snapshot_index(p->T, snapS));
    else if (mode == ELECTRIC)
      sprintf(fname, "director_field_%ld.csv", snapshot_index(p->elecE, snapS));
    else
      sprintf(fname, "director_field_%d.csv", p->first_file + it);
    print_n(fname, ni, *p, pt);
    if (mode == THERMAL)
      fprintf(po, "%g %g %g %g %g", p->T, S1, S2 - S1 * S1, E, E2 - E * E);
    else if (mode == ELECTRIC)
      fprintf(po, "%g %g %g %g %g", p->elecE, S1, S2 - S1 * S1, E, E2 - E * E);
    else
      fprintf(po, "%d %g %g %g %g", p->first_file + it, S1, S2 - S1 * S1, E, E2 - E * E);
    extra.write_values(po, p->MCS);
    fflush(po);
  }
  fclose(po);
  ok(mcl_destroy(e));
  return 0;
}

}  // namespace

thermalEvolveNGPU::thermalEvolveNGPU(float *ni, int *pt, Parameters *params) : EvolveNGPU(ni, pt, params) {}
thermalEvolveNGPU::~thermalEvolveNGPU() {}
int thermalEvolveNGPU::run() { return run_mode(THERMAL, ni, pt, params, geometry); }

stepEvolveNGPU::stepEvolveNGPU(float *ni, int *pt, Parameters *params) : EvolveNGPU(ni, pt, params) {}
stepEvolveNGPU::~stepEvolveNGPU() {}
int stepEvolveNGPU::run() { return run_mode(STEP, ni, pt, params, geometry); }

quenchEvolveNGPU::quenchEvolveNGPU(float *ni, int *pt, Parameters *params) : EvolveNGPU(ni, pt, params) {}
quenchEvolveNGPU::~quenchEvolveNGPU() {}
int quenchEvolveNGPU::run() { return run_mode(QUENCH, ni, pt, params, geometry); }

electricEvolveNGPU::electricEvolveNGPU(float *ni, int *pt, Parameters *params) : EvolveNGPU(ni, pt, params) {}
electricEvolveNGPU::~electricEvolveNGPU() {}
int electricEvolveNGPU::run() { return run_mode(ELECTRIC, ni, pt, params, geometry); }
