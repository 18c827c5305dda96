// ref_timing — times the reference's own CPU sweep (compiled from the reference sources with the GSL shim) on
// the host cores. Test/baseline infrastructure only.
//
//   mclics_ref_timing <input_file> <warmup> <steps> <measure 0|1> [noise seed [directors.f32]]
//
// Set-up as src/main.cpp:86-107 + src/simulator.cpp:32-126 (through the reference's functions). If `noise` > 0
// the initial directors get uniform noise of that amplitude per component and are renormalised (the C2 initial
// state "(0,0,1) + noise"), drawn from a splitmix64 stream of `seed`, instead of reading a CSV file. A raw file of
// 3 Nt float32 (the reference layout, x fastest) replaces the initial directors of the non-empty sites: the GPU
// arm of bench.py passes its own initial state this way, so both arms start from the same directors.
// One step = EvolveN::Monte_Carlo_Step (src/evolve.cpp:85-221) and, with measure = 1, the measurement the
// reference's mode loops do after each measurement sweep: energy_calculator + Q_tensor +
// Eigen_value_evaluation (src/evolve_thermal.cpp:95-102). The steps run at T = Ti and, in the electric mode, at the
// field Ei (one scan point of any mode). Prints one JSON line with the wall time of the timed
// steps, the thread count (OMP_NUM_THREADS or all cores) and the site count.
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <chrono>
#include <vector>

#include "../include/define.h"
#include "../include/evolve.h"
#include "../include/geometry.h"
#include "../include/ic.h"
#include "../include/io.h"
#include "../include/parameter_order.h"
#include "../include/parameters.h"
#include "../include/potential.h"
#include "gsl/gsl_rng.h"

struct TimedEvolve : public EvolveN {
  TimedEvolve(float *ni, int *pt, Parameters *p) : EvolveN(ni, pt, p) {}
};

static uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int main(int argc, char **argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s input warmup steps measure [noise seed]\n", argv[0]);
    return 2;
  }
  const int warmup = atoi(argv[2]), steps = atoi(argv[3]), measure = atoi(argv[4]);
  const double noise = argc > 5 ? atof(argv[5]) : 0.0;
  uint64_t nseed = argc > 6 ? strtoull(argv[6], 0, 0) : 7;

  Parameters params = read_input_file(argv[1]);
  params.flipMove = (strcasecmp(params.potential, "pear") == 0 || params.elecP != 0) ? 1 : 0;
  if (params.radial[0] == '\0') strcpy(params.radial, strcasecmp(params.geometry, "sphere") == 0 ? "sphere" : "none");
  if (params.elecA != 0 || params.elecP != 0) {
    float norm = sqrtf(params.elecX * params.elecX + params.elecY * params.elecY + params.elecZ * params.elecZ);
    params.elecX /= norm;
    params.elecY /= norm;
    params.elecZ /= norm;
  }
  validate_parameters(params);
  const int Nx = params.Nx, Ny = params.Ny, Nz = params.Nz;
  const long long Nt = (long long)Nx * Ny * Nz;
  float *ni = (float *)calloc(3 * Nt, sizeof(float));
  int *pt = (int *)calloc(3 * Nt, sizeof(int));
  TimedEvolve *ev = new TimedEvolve(ni, pt, &params);
  if (strcasecmp(params.geometry, "bulk") == 0)
    ev->geometry = new Bulk_Geometry(pt, &params);
  else if (strcasecmp(params.geometry, "slab") == 0)
    ev->geometry = new Slab_Geometry(pt, &params);
  else if (strcasecmp(params.geometry, "sphere") == 0)
    ev->geometry = new Sphere_Geometry(pt, &params);
  else
    ev->geometry = new Custom_Geometry(pt, &params);
  params.XBound = strcasecmp(params.XBoundtype, "periodic") == 0 ? &Periodic_Boundary : &Free_Boundary;
  params.YBound = strcasecmp(params.YBoundtype, "periodic") == 0 ? &Periodic_Boundary : &Free_Boundary;
  params.ZBound = strcasecmp(params.ZBoundtype, "periodic") == 0 ? &Periodic_Boundary : &Free_Boundary;
  check_checkerboard(params);
  ev->geometry->Boundary_Init(&params);
  apply_Initial_Conditions(ni, pt, params);
  if (noise > 0) {
    for (long long q = 0; q < Nt; q++) {
      if (!pt[q]) continue;
      double v[3];
      for (int c = 0; c < 3; c++) v[c] = ni[3 * q + c] + noise * (2.0 * ((splitmix64(nseed) >> 11) * 0x1.0p-53) - 1.0);
      double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (int c = 0; c < 3; c++) ni[3 * q + c] = (float)(v[c] / n);
    }
  }
  if (argc > 7) {
    FILE *f = fopen(argv[7], "rb");
    std::vector<float> v(3 * Nt);
    if (!f || fread(v.data(), sizeof(float), v.size(), f) != v.size()) {
      fprintf(stderr, "cannot read %lld directors from %s\n", Nt, argv[7]);
      return 2;
    }
    fclose(f);
    for (long long q = 0; q < Nt; q++)
      if (pt[q])
        for (int c = 0; c < 3; c++) ni[3 * q + c] = v[3 * q + c];
  }
  if (strcasecmp(params.potential, "ll") * strcasecmp(params.potential, "lebwohl-lasher") == 0) {
    ev->geometry->bulk_potential = &Bulk_Energy_Lebwohl_Lasher;
  } else if (strcasecmp(params.potential, "ghrl") * strcasecmp(params.potential, "gruhn-hess") == 0) {
    ev->geometry->bulk_potential = &Bulk_Energy_GHRL;
    setGHRL(params);
  } else {
    ev->geometry->bulk_potential = &Bulk_Energy_Selinger_Pear;
  }
  params.T = params.Ti;
  // the electric mode's first scan point (src/evolve_electric.cpp:67: elecE = Ei at the first field value); the
  // other modes keep elecE = 1
  if (strcasecmp(params.evol, "electric") == 0) params.elecE = params.elecEi;

  const int threads = omp_get_max_threads();
  gsl_rng **rng = (gsl_rng **)calloc(threads, sizeof(gsl_rng *));
  for (int i = 0; i < threads; i++) {
    rng[i] = gsl_rng_alloc(gsl_rng_ranlxs0);
    gsl_rng_set(rng[i], params.seed * 104729 + i);
  }
  float ang_var = 0.5f, mat[9], vec[3];
  double Esum = 0, Ssum = 0;
  auto step = [&]() {
    ev->Monte_Carlo_Step(ang_var, rng);
    if (measure) {
      Esum += ev->energy_calculator();
      Q_tensor(ni, mat, pt, params);
      Ssum += Eigen_value_evaluation(mat, vec);
    }
  };
  for (int s = 0; s < warmup; s++) step();
  auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < steps; s++) step();
  auto t1 = std::chrono::steady_clock::now();
  const double sec = std::chrono::duration<double>(t1 - t0).count();
  printf("{\"steps\": %d, \"seconds\": %.6f, \"threads\": %d, \"sites\": %lld, \"measure\": %d, "
         "\"ns_per_site_update\": %.4f, \"E_mean\": %.6f, \"S_mean\": %.6f, \"ang_var\": %.6f}\n",
         steps, sec, threads, Nt, measure, steps ? 1e9 * sec / ((double)steps * Nt) : 0.0,
         measure && (warmup + steps) ? Esum / (warmup + steps) : 0.0, measure && (warmup + steps) ? Ssum / (warmup + steps) : 0.0,
         ang_var);
  return 0;
}
