/* mc_oracle — CPU restatement of McLics' Metropolis sweep, site energies and observables.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load this library, and only as the checker. The CUDA library never calls it.
 *
 * Arithmetic mirrors the reference CPU code type for type (float terms, double bond accumulators and
 * double literals where the reference has them), so that with the same random numbers it reproduces the
 * reference bit for bit; compile with -ffp-contract=off. Pinned against the reference's own sources
 * compiled here (oracle/_ref, replay driver) by tests/test_oracle_pin.py.
 *
 * Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11), keyed by the replica seed and counted by (site, sweep, stream). The CUDA kernels use the same
 * function, so both sides see identical draws for a given (seed, sweep, site). */
#ifndef MC_ORACLE_H_
#define MC_ORACLE_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { MCO_POT_LL = 0, MCO_POT_GHRL = 1, MCO_POT_PEAR = 2 };
/* anchoring types, same numbering as the CUDA library's MCL_ANCH_* */
enum {
  MCO_ANCH_HOMEOTROPIC = 0,
  MCO_ANCH_RP = 1,
  MCO_ANCH_RP_TANGENT = 2,
  MCO_ANCH_FG = 3,
  MCO_ANCH_HOMEOTROPIC_GHRL = 4,
  MCO_ANCH_RP_GHRL = 5,
  MCO_ANCH_FG_GHRL = 6
};
enum { MCO_SCHED_REF8 = 0, MCO_SCHED_CHECKER2 = 1 };
#define MCO_MAX_SURFACES 16

typedef struct mco_model {
  int potential;
  float A, B1, C;
  float ghrl_lambda, ghrl_mu, ghrl_nu, ghrl_rho, ghrl_sigma;
  float field_dir[3]; /* unit vector (the reference normalises it in main.cpp:97-106) */
  float elecA, elecP, elecE;
  int flip_move;
  int n_surfaces;
  int anch_type[MCO_MAX_SURFACES];
  float anch_W[MCO_MAX_SURFACES];
  float anch_theta[MCO_MAX_SURFACES]; /* degrees (rp, rp_tangent, rp_ghrl) */
  float anch_phi[MCO_MAX_SURFACES];
} mco_model;

typedef struct mco_lattice {
  int nx, ny, nz;
  int periodic[3];
  const int *pt;   /* point types, Nx*Ny*Nz (0 empty, 1 bulk, s+2 surface s) */
  const float *ns; /* outward normals, 3 per site (AoS, reference layout) */
} mco_lattice;

/* Philox4x32-10 block function. */
void mco_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The uniforms of site (x, y, z) in `sweep` for the plain move: u[0] angle, u[1] axis, u[2] rotation
 * acceptance, u[3] flip acceptance.
 *  flip models (flip != 0): one Philox call per site, counter (site, sweep lo, sweep hi, 0), u[k] = (out[k] >> 8)
 *    2^-24;
 *  other models: one call per pair of same-colour sites x and x ^ 2 of a row, counter (linear index of
 *    (x & ~2, y, z), sweep lo, sweep hi, 0); the site uses the 64-bit half h = (x >> 1) & 1 of the output, split
 *    into three 21-bit fields: u = field 2^-21; u[3] = 0. */
void mco_site_uniforms(uint64_t seed, uint64_t sweep, int x, int y, int z, int nx, int ny, int flip, double u[4]);
/* Random initial director of a site (Philox stream 2): see mc_oracle.c. */
void mco_random_director(uint64_t seed, uint32_t site, float out[3]);

/* Site energy of site idx with its director replaced by n (reference geometry*::site_energy). */
float mco_site_energy(const mco_model *m, const mco_lattice *L, const float *ni, int idx, const float n[3]);
/* The same energy evaluated in FP64 throughout (for the FP64 oracle of reduced observables). */
double mco_site_energy_fp64(const mco_model *m, const mco_lattice *L, const float *ni, int idx);

/* One sweep in place. schedule: MCO_SCHED_REF8 = the reference CPU's 8 sublattices (evolve.cpp:106-119),
 * MCO_SCHED_CHECKER2 = two colours by parity of i+j+k. Returns the number of accepted rotations and
 * adapts *ang_var exactly as evolve.cpp:211-220. decisions (optional, one byte per site): bit0 rotation
 * accepted, bit1 flip accepted, bit7 site updated. margin (optional, one float per site): smallest
 * |u - exp(-dE/T)| of the site's decisions (|dE| at T = 0). */
int64_t mco_sweep(const mco_model *m, const mco_lattice *L, float *ni, float T, float *ang_var, uint64_t seed,
                  uint64_t sweep, int schedule, uint8_t *decisions, float *margin);

/* The uniforms the reference CPU consumes in one sweep, in its call order with OMP_NUM_THREADS=1
 * (evolve.cpp:106-201): per visited site u1, u2, u3 [, u4 if flip_move]. Returns the count written
 * (at most cap). */
int64_t mco_ref8_stream(const mco_model *m, const mco_lattice *L, uint64_t seed, uint64_t sweep, double *out,
                        int64_t cap);

/* Reference energy_calculator (evolve.cpp:33-75): double sum of float site energies / nValid, as float. */
float mco_energy_ref(const mco_model *m, const mco_lattice *L, const float *ni);
/* Reference Q_tensor (parameter_order.cpp:40-71): float accumulation, row-major 3x3. */
void mco_q_tensor_ref(const mco_lattice *L, const float *ni, float Q[9]);

/* FP64 observables: out[0] = sum of FP64 site energies, out[1..6] = sum of (3 n n - I)/2 components
 * xx, xy, xz, yy, yz, zz, out[7..9] = sum of n, out[10] = number of non-empty sites. */
void mco_observables_fp64(const mco_model *m, const mco_lattice *L, const float *ni, double out[11]);
/* Largest eigenvalue of the symmetric matrix (xx, xy, xz, yy, yz, zz) and its eigenvector (Jacobi, FP64). */
double mco_largest_eigen(const double q6[6], double vec[3]);

/* Sum of the float site energies in FP64 (what the CUDA reduction computes), divided by nValid. */
double mco_energy_fp64sum(const mco_model *m, const mco_lattice *L, const float *ni);

#ifdef __cplusplus
}
#endif
#endif
