/* mc_oracle.c — CPU restatement of McLics' checkerboard Metropolis sweep (test infrastructure only; see
 * mc_oracle.h). Every function cites the reference lines it restates. Build with -ffp-contract=off: the
 * reference's x86-64 build has no FMA, and the replay pin is bit-exact. */
#include "mc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al., SC'11): 10 rounds of two 32x32->64 multiplies with the published
 * multipliers and Weyl key increments. */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void mco_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
    uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += PHILOX_W0;
    k1 += PHILOX_W1;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* The engine's draw convention (mclics_b200/csrc/common.cuh): key fixed per stream, the seed in the counter
 * (a, b, seed_lo, seed_hi + c_hi). */
#define PHILOX_KEY0 0x694C634Du
#define PHILOX_KEY1 0x30303242u
static void stream_draws(uint32_t a, uint32_t b, uint64_t seed, uint32_t c_hi, uint32_t stream, uint32_t o[4]) {
  const uint32_t ctr[4] = {a, b, (uint32_t)seed, (uint32_t)(seed >> 32) + c_hi};
  const uint32_t key[2] = {PHILOX_KEY0 + stream, PHILOX_KEY1};
  mco_philox4x32_10(ctr, key, o);
}

void mco_site_uniforms(uint64_t seed, uint64_t sweep, int x, int y, int z, int nx, int ny, int flip, double u[4]) {
  uint32_t o[4];
  if (flip) {
    stream_draws((uint32_t)x + (uint32_t)nx * ((uint32_t)y + (uint32_t)ny * (uint32_t)z), (uint32_t)sweep, seed,
                 (uint32_t)(sweep >> 32), 0, o);
    for (int k = 0; k < 4; k++) u[k] = (double)(o[k] >> 8) * (1.0 / 16777216.0);
    return;
  }
  stream_draws(((uint32_t)x & ~2u) + (uint32_t)nx * ((uint32_t)y + (uint32_t)ny * (uint32_t)z), (uint32_t)sweep, seed,
               (uint32_t)(sweep >> 32), 0, o);
  const int h = (x >> 1) & 1;
  const uint32_t lo = o[2 * h], hi = o[2 * h + 1];
  const double s21 = 1.0 / 2097152.0;
  u[0] = (double)(lo & 0x1FFFFFu) * s21;
  u[1] = (double)(((lo >> 21) | (hi << 11)) & 0x1FFFFFu) * s21;
  u[2] = (double)((hi >> 10) & 0x1FFFFFu) * s21;
  u[3] = 0;
}

/* Random initial director of a site (the engine's `ic random` on the device, Philox stream 2; the reference
 * draws gsl_ran_dir_3d from a taus generator instead, src/ic.cpp:38-65, so parity with it is statistical): the
 * first draw (site, attempt) whose odd-integer grid point lies inside the ball of radius 2^24, projected onto the
 * unit sphere with one double square root and three double divisions. */
void mco_random_director(uint64_t seed, uint32_t site, float out[3]) {
  for (uint32_t attempt = 0; attempt < 64; attempt++) {
    uint32_t o[4];
    stream_draws(site, attempt, seed, 0, 2, o);
    const int64_t ix = 2 * (int64_t)(o[0] >> 8) + 1 - 16777216, iy = 2 * (int64_t)(o[1] >> 8) + 1 - 16777216,
                  iz = 2 * (int64_t)(o[2] >> 8) + 1 - 16777216;
    const int64_t s = ix * ix + iy * iy + iz * iz;
    if (s < ((int64_t)1 << 48)) {
      const double len = sqrt((double)s);
      out[0] = (float)((double)ix / len);
      out[1] = (float)((double)iy / len);
      out[2] = (float)((double)iz / len);
      return;
    }
  }
  out[0] = 0.f;
  out[1] = 0.f;
  out[2] = 1.f;
}

/* ------------------------------------------------------------------------------------------------ */
/* Pair potentials, reference potential.cpp (CPU), with its float/double typing. */

/* potential.cpp:28-31: -A * 1.5 * (ni.nj)^2, the product evaluated in double. */
static float pot_ll(const mco_model *m, const float ni[3], const float nj[3]) {
  float nij = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  return (float)((double)(-m->A) * 1.5 * (double)nij * (double)nij);
}

/* potential.cpp:40-56 (GHRL). E1 and the 1/9 and final sums are double, as in the reference. */
static float pot_ghrl(const mco_model *m, const float ni[3], const float nj[3], const float r[3]) {
  const float el = m->ghrl_lambda, em = m->ghrl_mu, en = m->ghrl_nu, er = m->ghrl_rho, es = m->ghrl_sigma;
  float ai = ni[0] * r[0] + ni[1] * r[1] + ni[2] * r[2];
  float aj = nj[0] * r[0] + nj[1] * r[1] + nj[2] * r[2];
  float nij = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  float pij = 1.5f * nij * nij - 0.5f;
  float cross = (ni[2] * nj[1] - ni[1] * nj[2]) * r[0] + (ni[0] * nj[2] - ni[2] * nj[0]) * r[1] +
                (ni[1] * nj[0] - ni[0] * nj[1]) * r[2];
  float E1 = (float)((1.5 * (double)ai * (double)ai) + (1.5 * (double)aj * (double)aj) - 1);
  float t1 = E1 * (er * pij + el);
  float t2 = ai * aj * nij;
  double acc = (double)t1 + (double)em * ((double)t2 - 1.0 / 9);
  acc = acc + (double)(en * pij);
  float t4 = es * (float)(nij > 0 ? 1 : -1) * cross;
  acc = acc + (double)t4;
  return (float)acc;
}

/* potential.cpp:19-24 (pear, Dhakal & Selinger). */
static float pot_pear(const mco_model *m, const float ni[3], const float nj[3], const float r[3]) {
  float nij = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  float polar_splay =
      (1 + 2 * nij + nij * nij) * ((nj[0] - ni[0]) * r[0] + (nj[1] - ni[1]) * r[1] + (nj[2] - ni[2]) * r[2]);
  float f = -m->A * nij * nij - m->B1 * nij;
  return (float)((double)f - ((double)m->C * 0.25) * (double)polar_splay);
}

static float pot(const mco_model *m, const float ni[3], const float nj[3], const float r[3]) {
  switch (m->potential) {
    case MCO_POT_GHRL: return pot_ghrl(m, ni, nj, r);
    case MCO_POT_PEAR: return pot_pear(m, ni, nj, r);
    default: return pot_ll(m, ni, nj);
  }
}

/* potential.cpp:59-63 (field term, elecE = current magnitude). */
static float pot_field(const mco_model *m, const float n[3]) {
  float nDotE = m->elecE * (n[0] * m->field_dir[0] + n[1] * m->field_dir[1] + n[2] * m->field_dir[2]);
  return -m->elecP * nDotE - m->elecA * nDotE * nDotE;
}

/* anchoring.cpp:19-24 */
static void lab_axis(float theta_deg, float phi_deg, float out[3]) {
  const float toRad = (float)(M_PI / 180);
  out[0] = sinf(toRad * theta_deg) * cosf(toRad * phi_deg);
  out[1] = sinf(toRad * theta_deg) * sinf(toRad * phi_deg);
  out[2] = cosf(toRad * theta_deg);
}

/* anchoring_{homeotropic,rp,rp_tangent,fg}.cpp surface_potential (energy including W). */
static float anchoring(const mco_model *m, int s_id, const float n[3], const float s[3]) {
  const float W = m->anch_W[s_id];
  float e[3], nij;
  switch (m->anch_type[s_id]) {
    case MCO_ANCH_HOMEOTROPIC: /* anchoring_homeotropic.cpp:20-23 */
      nij = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
      return -W * nij * nij;
    case MCO_ANCH_RP: /* anchoring_rp.cpp:33-36 */
      lab_axis(m->anch_theta[s_id], m->anch_phi[s_id], e);
      nij = n[0] * e[0] + n[1] * e[1] + n[2] * e[2];
      return -W * nij * nij;
    case MCO_ANCH_RP_TANGENT: { /* anchoring_rp_tangent.cpp:49-70 */
      float d[3];
      lab_axis(m->anch_theta[s_id], m->anch_phi[s_id], d);
      float ds = d[0] * s[0] + d[1] * s[1] + d[2] * s[2];
      e[0] = d[0] - ds * s[0];
      e[1] = d[1] - ds * s[1];
      e[2] = d[2] - ds * s[2];
      float mod = sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
      if (mod < 1e-3f) return 0;
      e[0] /= mod;
      e[1] /= mod;
      e[2] /= mod;
      nij = n[0] * e[0] + n[1] * e[1] + n[2] * e[2];
      return -W * nij * nij;
    }
    case MCO_ANCH_FG: /* anchoring_fg.cpp:17-20 */
      nij = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
      return +W * nij * nij;
    case MCO_ANCH_HOMEOTROPIC_GHRL: /* anchoring_homeotropic.cpp:37-40 */
      return W * pot_ghrl(m, n, s, s);
    case MCO_ANCH_RP_GHRL: /* anchoring_rp.cpp:62-65 */
      lab_axis(m->anch_theta[s_id], m->anch_phi[s_id], e);
      return W * pot_ghrl(m, n, e, s);
    case MCO_ANCH_FG_GHRL: { /* anchoring_fg.cpp:37-47 */
      float ns = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
      float nj[3] = {n[0] - ns * s[0], n[1] - ns * s[1], n[2] - ns * s[2]};
      float mod = sqrtf(nj[0] * nj[0] + nj[1] * nj[1] + nj[2] * nj[2]);
      if (mod < 1e-6f) return 0;
      nj[0] /= mod;
      nj[1] /= mod;
      nj[2] /= mod;
      return W * pot_ghrl(m, n, nj, s);
    }
  }
  return 0;
}

/* potential.cpp:64-74: periodic wraps, free marks the neighbour beyond the edge as absent. */
static int bound(int periodic, int *ii, int N) {
  if (periodic) {
    *ii = (*ii + N) % N;
    return 1;
  }
  return !(*ii == -1 || *ii == N);
}

static int pt_of(const mco_lattice *L, int idx) { return L->pt ? L->pt[idx] : 1; }

/* geometry.cpp:23-76 (bond sum in double) + geometry_{bulk,slab,sphere,custom}.cpp site_energy. */
float mco_site_energy(const mco_model *m, const mco_lattice *L, const float *ni, int idx, const float n[3]) {
  const int Nx = L->nx, Ny = L->ny, Nz = L->nz;
  const int i = idx % Nx, j = (idx / Nx) % Ny, k = idx / (Nx * Ny);
  static const float dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  double E = 0;
  for (int d = 0; d < 6; d++) {
    int ii = i + (int)dirs[d][0], jj = j + (int)dirs[d][1], kk = k + (int)dirs[d][2];
    int ok;
    if (d < 2)
      ok = bound(L->periodic[0], &ii, Nx);
    else if (d < 4)
      ok = bound(L->periodic[1], &jj, Ny);
    else
      ok = bound(L->periodic[2], &kk, Nz);
    if (!ok) continue;
    int jdx = ii + Nx * (jj + Ny * kk);
    if (!pt_of(L, jdx)) continue;
    E += pot(m, n, &ni[3 * jdx], dirs[d]);
  }
  float Ef = (float)E;
  int p = pt_of(L, idx);
  if (p > 1 && L->ns) Ef += anchoring(m, p - 2, n, &L->ns[3 * idx]);
  if (m->elecA != 0 || m->elecP != 0) Ef += pot_field(m, n);
  return Ef;
}

/* ---- FP64 versions of the same formulas (no reference counterpart: the FP64 oracle for reductions) ---- */
static double dot3d(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static double pot_fp64(const mco_model *m, const double a[3], const double b[3], const double r[3]) {
  double nij = dot3d(a, b);
  if (m->potential == MCO_POT_LL) return -(double)m->A * 1.5 * nij * nij;
  if (m->potential == MCO_POT_PEAR) {
    double ps = (1 + 2 * nij + nij * nij) * ((b[0] - a[0]) * r[0] + (b[1] - a[1]) * r[1] + (b[2] - a[2]) * r[2]);
    return -(double)m->A * nij * nij - (double)m->B1 * nij - (double)m->C * 0.25 * ps;
  }
  double ai = dot3d(a, r), aj = dot3d(b, r);
  double pij = 1.5 * nij * nij - 0.5;
  double cross = (a[2] * b[1] - a[1] * b[2]) * r[0] + (a[0] * b[2] - a[2] * b[0]) * r[1] + (a[1] * b[0] - a[0] * b[1]) * r[2];
  double E1 = 1.5 * ai * ai + 1.5 * aj * aj - 1;
  return E1 * (m->ghrl_rho * pij + m->ghrl_lambda) + m->ghrl_mu * (ai * aj * nij - 1.0 / 9) + m->ghrl_nu * pij +
         m->ghrl_sigma * (nij > 0 ? 1.0 : -1.0) * cross;
}

static double anchoring_fp64(const mco_model *m, int s_id, const double n[3], const double s[3]) {
  const double W = m->anch_W[s_id];
  double e[3], nij;
  const double toRad = M_PI / 180;
  double th = m->anch_theta[s_id] * toRad, ph = m->anch_phi[s_id] * toRad;
  double lab[3] = {sin(th) * cos(ph), sin(th) * sin(ph), cos(th)};
  switch (m->anch_type[s_id]) {
    case MCO_ANCH_HOMEOTROPIC: nij = dot3d(n, s); return -W * nij * nij;
    case MCO_ANCH_RP: nij = dot3d(n, lab); return -W * nij * nij;
    case MCO_ANCH_RP_TANGENT: {
      double ds = dot3d(lab, s);
      for (int c = 0; c < 3; c++) e[c] = lab[c] - ds * s[c];
      double mod = sqrt(dot3d(e, e));
      if (mod < 1e-3) return 0;
      for (int c = 0; c < 3; c++) e[c] /= mod;
      nij = dot3d(n, e);
      return -W * nij * nij;
    }
    case MCO_ANCH_FG: nij = dot3d(n, s); return W * nij * nij;
    case MCO_ANCH_HOMEOTROPIC_GHRL: return W * pot_fp64(m, n, s, s);
    case MCO_ANCH_RP_GHRL: return W * pot_fp64(m, n, lab, s);
    case MCO_ANCH_FG_GHRL: {
      double ns = dot3d(n, s);
      for (int c = 0; c < 3; c++) e[c] = n[c] - ns * s[c];
      double mod = sqrt(dot3d(e, e));
      if (mod < 1e-6) return 0;
      for (int c = 0; c < 3; c++) e[c] /= mod;
      return W * pot_fp64(m, n, e, s);
    }
  }
  return 0;
}

double mco_site_energy_fp64(const mco_model *m, const mco_lattice *L, const float *ni, int idx) {
  const int Nx = L->nx, Ny = L->ny, Nz = L->nz;
  const int i = idx % Nx, j = (idx / Nx) % Ny, k = idx / (Nx * Ny);
  static const double dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  double n[3] = {ni[3 * idx], ni[3 * idx + 1], ni[3 * idx + 2]};
  double E = 0;
  for (int d = 0; d < 6; d++) {
    int ii = i + (int)dirs[d][0], jj = j + (int)dirs[d][1], kk = k + (int)dirs[d][2];
    int ok = d < 2 ? bound(L->periodic[0], &ii, Nx) : d < 4 ? bound(L->periodic[1], &jj, Ny) : bound(L->periodic[2], &kk, Nz);
    if (!ok) continue;
    int jdx = ii + Nx * (jj + Ny * kk);
    if (!pt_of(L, jdx)) continue;
    double b[3] = {ni[3 * jdx], ni[3 * jdx + 1], ni[3 * jdx + 2]};
    E += pot_fp64(m, n, b, dirs[d]);
  }
  int p = pt_of(L, idx);
  if (p > 1 && L->ns) {
    double s[3] = {L->ns[3 * idx], L->ns[3 * idx + 1], L->ns[3 * idx + 2]};
    E += anchoring_fp64(m, p - 2, n, s);
  }
  if (m->elecA != 0 || m->elecP != 0) {
    double nDotE = (double)m->elecE * (n[0] * m->field_dir[0] + n[1] * m->field_dir[1] + n[2] * m->field_dir[2]);
    E += -(double)m->elecP * nDotE - (double)m->elecA * nDotE * nDotE;
  }
  return E;
}

/* ------------------------------------------------------------------------------------------------ */
/* evolve.cpp:133-207: one trial move (rotation, then the optional n -> -n trial) of site (i, j, k). */
static int update_site(const mco_model *m, const mco_lattice *L, float *ni, int idx, float T, float ang_var,
                       uint64_t seed, uint64_t sweep, uint8_t *decisions, float *margin) {
  double u[4];
  const int x = idx % L->nx, y = (idx / L->nx) % L->ny, z = idx / (L->nx * L->ny);
  mco_site_uniforms(seed, sweep, x, y, z, L->nx, L->ny, m->flip_move, u);
  float *n = &ni[3 * idx];
  float va = (float)((2 * u[0] - 1) * (double)ang_var);
  float rotation_type = (float)u[1];
  float nNew[3];
  float c = cosf((float)(M_PI * (double)va)), s = sinf((float)(M_PI * (double)va));
  if ((double)rotation_type < 0.333) {
    nNew[0] = n[0];
    nNew[1] = n[1] * c + n[2] * s;
    nNew[2] = n[2] * c - n[1] * s;
  } else if ((double)rotation_type < 0.666) {
    nNew[0] = n[0] * c - n[2] * s;
    nNew[1] = n[1];
    nNew[2] = n[2] * c + n[0] * s;
  } else {
    nNew[0] = n[0] * c + n[1] * s;
    nNew[1] = n[1] * c - n[0] * s;
    nNew[2] = n[2];
  }
  float norm = sqrtf(nNew[0] * nNew[0] + nNew[1] * nNew[1] + nNew[2] * nNew[2]);
  nNew[0] /= norm;
  nNew[1] /= norm;
  nNew[2] /= norm;

  float cur[3] = {n[0], n[1], n[2]};
  float E_old = mco_site_energy(m, L, ni, idx, cur);
  float E_new = mco_site_energy(m, L, ni, idx, nNew);
  float E_cur = E_old;
  float uu = (float)u[2];
  int acc;
  float mg;
  if (T > 0) {
    float p = expf(-(E_new - E_old) / T);
    acc = uu < p;
    mg = fabsf(uu - p);
  } else {
    acc = E_new <= E_old;
    mg = fabsf(E_new - E_old);
  }
  uint8_t dec = 0x80;
  if (acc) {
    n[0] = nNew[0];
    n[1] = nNew[1];
    n[2] = nNew[2];
    E_cur = E_new;
    dec |= 1;
  }
  if (m->flip_move) {
    float f[3] = {-n[0], -n[1], -n[2]};
    float E_flip = mco_site_energy(m, L, ni, idx, f);
    float uf = (float)u[3];
    int accf;
    float mgf;
    if (T > 0) {
      float p = expf(-(E_flip - E_cur) / T);
      accf = uf < p;
      mgf = fabsf(uf - p);
    } else {
      accf = E_flip <= E_cur;
      mgf = fabsf(E_flip - E_cur);
    }
    if (mgf < mg) mg = mgf;
    if (accf) {
      n[0] = f[0];
      n[1] = f[1];
      n[2] = f[2];
      dec |= 2;
    }
  }
  if (decisions) decisions[idx] = dec;
  if (margin) margin[idx] = mg;
  return acc;
}

/* evolve.cpp:211-220 */
static void adapt(float *ang_var, int64_t acceptance, int64_t nValid) {
  if (1.0 * acceptance / nValid < 0.5) {
    *ang_var = (float)((double)*ang_var * 0.99);
    if (*ang_var < 0.01) *ang_var = 0.01f;
  } else if (1.0 * acceptance / nValid > 0.5) {
    *ang_var = (float)((double)*ang_var / 0.99);
    if (*ang_var > 1.0) *ang_var -= 0.5f;
  }
}

int64_t mco_sweep(const mco_model *m, const mco_lattice *L, float *ni, float T, float *ang_var, uint64_t seed,
                  uint64_t sweep, int schedule, uint8_t *decisions, float *margin) {
  const int Nx = L->nx, Ny = L->ny, Nz = L->nz;
  const int64_t Nt = (int64_t)Nx * Ny * Nz;
  int64_t nValid = 0, acceptance = 0;
  for (int64_t q = 0; q < Nt; q++) nValid += pt_of(L, (int)q) ? 1 : 0;
  if (decisions && Nt > 0) memset(decisions, 0, (size_t)Nt);
  if (margin)
    for (int64_t q = 0; q < Nt; q++) margin[q] = INFINITY;
  const float av = *ang_var;
  if (schedule == MCO_SCHED_REF8) {
    const int nBoxX = Nx / 2 + Nx % 2, nBoxY = Ny / 2 + Ny % 2, nBoxZ = Nz / 2 + Nz % 2;
    const int64_t Ntt = (int64_t)nBoxX * nBoxY * nBoxZ;
    for (int tick = 0; tick < 8; tick++) {
      int di = tick % 2, dj = (tick / 2) % 2, dk = tick / 4;
      for (int64_t nt = 0; nt < Ntt; nt++) {
        int iBox = (int)(nt % nBoxX), jBox = (int)((nt / nBoxX) % nBoxY), kBox = (int)(nt / nBoxX / nBoxY);
        int i = di + 2 * iBox, j = dj + 2 * jBox, k = dk + 2 * kBox;
        if (i >= Nx || j >= Ny || k >= Nz) continue;
        int idx = i + Nx * (j + Ny * k);
        if (!pt_of(L, idx)) continue;
        acceptance += update_site(m, L, ni, idx, T, av, seed, sweep, decisions, margin);
      }
    }
  } else {
    for (int colour = 0; colour < 2; colour++)
      for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++)
          for (int i = 0; i < Nx; i++) {
            if (((i + j + k) & 1) != colour) continue;
            int idx = i + Nx * (j + Ny * k);
            if (!pt_of(L, idx)) continue;
            acceptance += update_site(m, L, ni, idx, T, av, seed, sweep, decisions, margin);
          }
  }
  adapt(ang_var, acceptance, nValid);
  return acceptance;
}

int64_t mco_ref8_stream(const mco_model *m, const mco_lattice *L, uint64_t seed, uint64_t sweep, double *out,
                        int64_t cap) {
  const int Nx = L->nx, Ny = L->ny, Nz = L->nz;
  const int nBoxX = Nx / 2 + Nx % 2, nBoxY = Ny / 2 + Ny % 2, nBoxZ = Nz / 2 + Nz % 2;
  const int64_t Ntt = (int64_t)nBoxX * nBoxY * nBoxZ;
  int64_t w = 0;
  for (int tick = 0; tick < 8; tick++) {
    int di = tick % 2, dj = (tick / 2) % 2, dk = tick / 4;
    for (int64_t nt = 0; nt < Ntt; nt++) {
      int iBox = (int)(nt % nBoxX), jBox = (int)((nt / nBoxX) % nBoxY), kBox = (int)(nt / nBoxX / nBoxY);
      int i = di + 2 * iBox, j = dj + 2 * jBox, k = dk + 2 * kBox;
      if (i >= Nx || j >= Ny || k >= Nz) continue;
      int idx = i + Nx * (j + Ny * k);
      if (!pt_of(L, idx)) continue;
      double u[4];
      mco_site_uniforms(seed, sweep, i, j, k, Nx, Ny, m->flip_move, u);
      int n = m->flip_move ? 4 : 3;
      for (int q = 0; q < n; q++) {
        if (w < cap) out[w] = u[q];
        w++;
      }
    }
  }
  return w;
}

/* evolve.cpp:33-75 */
float mco_energy_ref(const mco_model *m, const mco_lattice *L, const float *ni) {
  const int64_t Nt = (int64_t)L->nx * L->ny * L->nz;
  int64_t nValid = 0;
  double Etot = 0;
  for (int64_t q = 0; q < Nt; q++) {
    if (!pt_of(L, (int)q)) continue;
    nValid++;
    Etot += mco_site_energy(m, L, ni, (int)q, &ni[3 * q]);
  }
  return (float)(Etot / nValid);
}

double mco_energy_fp64sum(const mco_model *m, const mco_lattice *L, const float *ni) {
  const int64_t Nt = (int64_t)L->nx * L->ny * L->nz;
  int64_t nValid = 0;
  double Etot = 0;
  for (int64_t q = 0; q < Nt; q++) {
    if (!pt_of(L, (int)q)) continue;
    nValid++;
    Etot += (double)mco_site_energy(m, L, ni, (int)q, &ni[3 * q]);
  }
  return Etot / (double)nValid;
}

/* parameter_order.cpp:40-71 (x outermost, float accumulators, double per-term arithmetic). */
void mco_q_tensor_ref(const mco_lattice *L, const float *ni, float Q[9]) {
  const int Nx = L->nx, Ny = L->ny, Nz = L->nz;
  int points = 0;
  for (int q = 0; q < 9; q++) Q[q] = 0;
  for (int i = 0; i < Nx; i++)
    for (int j = 0; j < Ny; j++)
      for (int k = 0; k < Nz; k++) {
        int idx = i + Nx * (j + Ny * k);
        if (!pt_of(L, idx)) continue;
        const float *n = &ni[3 * idx];
        Q[0] = (float)((double)Q[0] + (3.0 * (double)(n[0] * n[0]) - 1));
        Q[1] = (float)((double)Q[1] + 3.0 * (double)(n[0] * n[1]));
        Q[2] = (float)((double)Q[2] + 3.0 * (double)(n[0] * n[2]));
        Q[4] = (float)((double)Q[4] + (3.0 * (double)(n[1] * n[1]) - 1));
        Q[5] = (float)((double)Q[5] + 3.0 * (double)(n[1] * n[2]));
        points++;
      }
  Q[0] = (float)(Q[0] / (2.0 * points));
  Q[1] = (float)(Q[1] / (2.0 * points));
  Q[2] = (float)(Q[2] / (2.0 * points));
  Q[4] = (float)(Q[4] / (2.0 * points));
  Q[5] = (float)(Q[5] / (2.0 * points));
  Q[3] = Q[1];
  Q[6] = Q[2];
  Q[7] = Q[5];
  Q[8] = -Q[0] - Q[4];
}

void mco_observables_fp64(const mco_model *m, const mco_lattice *L, const float *ni, double out[11]) {
  const int64_t Nt = (int64_t)L->nx * L->ny * L->nz;
  for (int q = 0; q < 11; q++) out[q] = 0;
  for (int64_t q = 0; q < Nt; q++) {
    if (!pt_of(L, (int)q)) continue;
    double x = ni[3 * q], y = ni[3 * q + 1], z = ni[3 * q + 2];
    out[0] += mco_site_energy_fp64(m, L, ni, (int)q);
    out[1] += 1.5 * x * x - 0.5;
    out[2] += 1.5 * x * y;
    out[3] += 1.5 * x * z;
    out[4] += 1.5 * y * y - 0.5;
    out[5] += 1.5 * y * z;
    out[6] += 1.5 * z * z - 0.5;
    out[7] += x;
    out[8] += y;
    out[9] += z;
    out[10] += 1;
  }
}

/* Cyclic Jacobi on a 3x3 symmetric matrix (Golub & Van Loan, Algorithm 8.5.3); returns the largest
 * eigenvalue (parameter_order.cpp:19-37 takes the first after a descending sort). */
double mco_largest_eigen(const double q6[6], double vec[3]) {
  double a[3][3] = {{q6[0], q6[1], q6[2]}, {q6[1], q6[3], q6[4]}, {q6[2], q6[4], q6[5]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-34 * dg || off == 0) break;
    for (int p = 0; p < 3; p++)
      for (int q = p + 1; q < 3; q++) {
        double apq = a[p][q];
        if (apq == 0) continue;
        double theta = (a[q][q] - a[p][p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        double c = 1 / sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 3; k++) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; k++) {
          double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int best = 0;
  for (int q = 1; q < 3; q++)
    if (a[q][q] > a[best][best]) best = q;
  if (vec)
    for (int k = 0; k < 3; k++) vec[k] = v[k][best];
  return a[best][best];
}
