// Site energies and the trial move for the production kernels: FP32, explicit fmaf everywhere it matters, so
// that every kernel that calls these functions (untiled and fused) rounds identically.
//
// Definitions follow the reference CPU code (src/potential.cpp:19-63, src/anchoring_*.cpp,
// src/geometry*.cpp site_energy): E_site = sum over present neighbours of U(n, n_j, r_j) + [surface] anchoring
// + [elecA or elecP != 0] field. Neighbour order +x, -x, +y, -y, +z, -z (src/geometry.cpp:23-76); the bond vector
// r_j is a compile-time unit vector here, so its zero components cost nothing. An absent neighbour has weight 0.
#pragma once
#include "common.cuh"

namespace mcl {

struct Vec3 {
  float x, y, z;
};
__device__ __forceinline__ float dot(const Vec3 &a, const Vec3 &b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ float comp(const Vec3 &a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }

// Bond D = 0..5 is +x, -x, +y, -y, +z, -z: axis D/2, sign +1 for even D.
template <int D>
struct BondDir {
  static constexpr int axis = D / 2;
  static constexpr float sign = (D % 2 == 0) ? 1.f : -1.f;
};

// Lebwohl-Lasher, src/potential.cpp:28-31: -1.5 A (n.n_j)^2.
__device__ __forceinline__ float ll_bond(const ModelDev &m, const Vec3 &x, const Vec3 &y) {
  const float b = dot(x, y);
  return __fmul_rn(-1.5f * m.A, __fmul_rn(b, b));
}

// GHRL with bond vector r = sign * e_axis, src/potential.cpp:40-56.
template <int AXIS>
__device__ __forceinline__ float ghrl_bond(const ModelDev &m, const Vec3 &x, const Vec3 &y, float sign) {
  const float ai = comp(x, AXIS), aj = comp(y, AXIS);  // a_i a_j and a^2 do not depend on the sign of r
  const float b = dot(x, y);
  const float p2 = fmaf(__fmul_rn(1.5f, b), b, -0.5f);
  const float e1 = fmaf(1.5f, fmaf(ai, ai, __fmul_rn(aj, aj)), -1.f);
  float u = fmaf(e1, fmaf(m.rho, p2, m.lam), fmaf(m.mu, fmaf(__fmul_rn(ai, aj), b, -1.f / 9.f), __fmul_rn(m.nu, p2)));
  if (m.sigma != 0.f) {
    // c = r . (n_j x n_i)
    const float c = AXIS == 0 ? fmaf(y.y, x.z, -__fmul_rn(y.z, x.y))
                              : (AXIS == 1 ? fmaf(y.z, x.x, -__fmul_rn(y.x, x.z)) : fmaf(y.x, x.y, -__fmul_rn(y.y, x.x)));
    u = fmaf(__fmul_rn(m.sigma * sign, b > 0.f ? 1.f : -1.f), c, u);
  }
  return u;
}

// GHRL with an arbitrary bond vector (anchoring phantom neighbour along the surface normal).
__device__ __forceinline__ float ghrl_general(const ModelDev &m, const Vec3 &x, const Vec3 &y, const Vec3 &r) {
  const float ai = dot(x, r), aj = dot(y, r), b = dot(x, y);
  const float p2 = fmaf(__fmul_rn(1.5f, b), b, -0.5f);
  const float e1 = fmaf(1.5f, fmaf(ai, ai, __fmul_rn(aj, aj)), -1.f);
  float u = fmaf(e1, fmaf(m.rho, p2, m.lam), fmaf(m.mu, fmaf(__fmul_rn(ai, aj), b, -1.f / 9.f), __fmul_rn(m.nu, p2)));
  if (m.sigma != 0.f) {
    const float c = fmaf(r.x, fmaf(y.y, x.z, -__fmul_rn(y.z, x.y)),
                         fmaf(r.y, fmaf(y.z, x.x, -__fmul_rn(y.x, x.z)), __fmul_rn(r.z, fmaf(y.x, x.y, -__fmul_rn(y.y, x.x)))));
    u = fmaf(__fmul_rn(m.sigma, b > 0.f ? 1.f : -1.f), c, u);
  }
  return u;
}

// Pear (Dhakal & Selinger), src/potential.cpp:19-24: -A b^2 - B1 b - C/4 (1+b)^2 r.(n_j - n_i).
template <int AXIS>
__device__ __forceinline__ float pear_bond(const ModelDev &m, const Vec3 &x, const Vec3 &y, float sign) {
  const float b = dot(x, y);
  const float opb = 1.f + b;
  const float ps = __fmul_rn(__fmul_rn(opb, opb), sign * (comp(y, AXIS) - comp(x, AXIS)));
  return fmaf(__fmul_rn(-m.A, b), b, fmaf(-m.B1, b, __fmul_rn(-0.25f * m.C, ps)));
}

template <int POT, int D>
__device__ __forceinline__ float bond(const ModelDev &m, const Vec3 &x, const Vec3 &y) {
  if (POT == POT_LL) return ll_bond(m, x, y);
  if (POT == POT_GHRL) return ghrl_bond<BondDir<D>::axis>(m, x, y, BondDir<D>::sign);
  return pear_bond<BondDir<D>::axis>(m, x, y, BondDir<D>::sign);
}

// Sum over the six bonds with weights w[d] in {0, 1} (0: free edge or empty site).
template <int POT>
__device__ __forceinline__ float bond_sum(const ModelDev &m, const Vec3 &x, const Vec3 (&nb)[6], const float (&w)[6]) {
  float e = __fmul_rn(w[0], bond<POT, 0>(m, x, nb[0]));
  e = fmaf(w[1], bond<POT, 1>(m, x, nb[1]), e);
  e = fmaf(w[2], bond<POT, 2>(m, x, nb[2]), e);
  e = fmaf(w[3], bond<POT, 3>(m, x, nb[3]), e);
  e = fmaf(w[4], bond<POT, 4>(m, x, nb[4]), e);
  e = fmaf(w[5], bond<POT, 5>(m, x, nb[5]), e);
  return e;
}

// Field, src/potential.cpp:59-63.
__device__ __forceinline__ float field_energy(const ModelDev &m, const Vec3 &x, float elecE) {
  const float ne = __fmul_rn(elecE, fmaf(x.x, m.fdir[0], fmaf(x.y, m.fdir[1], __fmul_rn(x.z, m.fdir[2]))));
  return fmaf(-m.elecA, __fmul_rn(ne, ne), __fmul_rn(-m.elecP, ne));
}

// Anchoring of surface sid for a site with outward normal s (src/anchoring_*.cpp surface_potential, W included).
__device__ __forceinline__ float anchoring_energy(const ModelDev &m, int sid, const Vec3 &x, const Vec3 &s) {
  const float W = m.anch_W[sid];
  const Vec3 lab{m.anch_lab[sid][0], m.anch_lab[sid][1], m.anch_lab[sid][2]};
  switch (m.anch_type[sid]) {
    case ANCH_HOMEOTROPIC: {
      const float c = dot(x, s);
      return __fmul_rn(-W, __fmul_rn(c, c));
    }
    case ANCH_RP: {
      const float c = dot(x, lab);
      return __fmul_rn(-W, __fmul_rn(c, c));
    }
    case ANCH_RP_TANGENT: {
      const float ds = dot(lab, s);
      const Vec3 e{fmaf(-ds, s.x, lab.x), fmaf(-ds, s.y, lab.y), fmaf(-ds, s.z, lab.z)};
      const float mod = sqrtf(dot(e, e));
      if (mod < 1e-3f) return 0.f;
      const float c = dot(x, e) / mod;
      return __fmul_rn(-W, __fmul_rn(c, c));
    }
    case ANCH_FG: {
      const float c = dot(x, s);
      return __fmul_rn(W, __fmul_rn(c, c));
    }
    case ANCH_HOMEOTROPIC_GHRL:
      return __fmul_rn(W, ghrl_general(m, x, s, s));
    case ANCH_RP_GHRL:
      return __fmul_rn(W, ghrl_general(m, x, lab, s));
    case ANCH_FG_GHRL: {
      const float c = dot(x, s);
      const Vec3 t{fmaf(-c, s.x, x.x), fmaf(-c, s.y, x.y), fmaf(-c, s.z, x.z)};
      const float mod = sqrtf(dot(t, t));
      if (mod < 1e-6f) return 0.f;
      const float inv = 1.f / mod;
      const Vec3 tn{__fmul_rn(t.x, inv), __fmul_rn(t.y, inv), __fmul_rn(t.z, inv)};
      return __fmul_rn(W, ghrl_general(m, x, tn, s));
    }
  }
  return 0.f;
}

// Single-site terms: anchoring (sid >= 0) and field.
__device__ __forceinline__ float single_energy(const ModelDev &m, const Vec3 &x, int sid, const Vec3 &s, float elecE) {
  float e = 0.f;
  if (sid >= 0) e = anchoring_energy(m, sid, x, s);
  if (m.field_on) e = __fadd_rn(e, field_energy(m, x, elecE));
  return e;
}

// Trial rotation by pi * va about axis `axis` (src/evolve.cpp:153-176): the reference's three rotations in one
// branch-free Rodrigues form n' = c n + (1 - c) n_a e_a - s (e_a x n), then renormalised.
__device__ __forceinline__ Vec3 rotate_trial(const Vec3 &n, float va, int axis) {
  float s, c;
  __sincosf(__fmul_rn(3.14159265358979f, va), &s, &c);  // |pi va| <= pi: the hardware sin/cos range
  const float w0 = axis == 0 ? 1.f : 0.f, w1 = axis == 1 ? 1.f : 0.f, w2 = axis == 2 ? 1.f : 0.f;
  const float cx = fmaf(w1, n.z, -__fmul_rn(w2, n.y)), cy = fmaf(w2, n.x, -__fmul_rn(w0, n.z)),
              cz = fmaf(w0, n.y, -__fmul_rn(w1, n.x));
  const float omc = 1.f - c;
  const Vec3 r{fmaf(c, n.x, fmaf(__fmul_rn(omc, w0), n.x, -__fmul_rn(s, cx))),
               fmaf(c, n.y, fmaf(__fmul_rn(omc, w1), n.y, -__fmul_rn(s, cy))),
               fmaf(c, n.z, fmaf(__fmul_rn(omc, w2), n.z, -__fmul_rn(s, cz)))};
  const float inv = rsqrtf(dot(r, r));
  return Vec3{__fmul_rn(r.x, inv), __fmul_rn(r.y, inv), __fmul_rn(r.z, inv)};
}

// Metropolis test u < exp(-dE/T); T = 0 accepts when the energy does not increase (src/evolve.cpp:185-188).
__device__ __forceinline__ bool metropolis(float u, float dE, float invT, float T) {
  return T > 0.f ? (u < __expf(-__fmul_rn(dE, invT))) : (dE <= 0.f);
}

// Result of one trial move of one site.
struct SiteResult {
  Vec3 n;          // director after the move
  float bond;      // bond energy of the final director
  float single;    // single-site energy of the final director
  unsigned rot;    // 1 if the rotation was accepted
  unsigned flip;   // 1 if the flip was accepted
};

// One trial move (src/evolve.cpp:133-207): rotation, Metropolis, then the optional n -> -n trial.
template <int POT, bool FLIP>
__device__ __forceinline__ SiteResult site_update(const ModelDev &m, const Vec3 &n, const Vec3 (&nb)[6],
                                                  const float (&w)[6], int sid, const Vec3 &s, float elecE,
                                                  const Draw &d, float av, float T, float invT) {
  const float va = __fmul_rn(fmaf(2.f, unif(d.f1, FLIP), -1.f), av);
  const Vec3 nn = rotate_trial(n, va, rotation_axis(d.f2, FLIP));
  const float b_old = bond_sum<POT>(m, n, nb, w), b_new = bond_sum<POT>(m, nn, nb, w);
  const float s_old = single_energy(m, n, sid, s, elecE), s_new = single_energy(m, nn, sid, s, elecE);
  const float e_old = __fadd_rn(b_old, s_old), e_new = __fadd_rn(b_new, s_new);
  SiteResult r;
  const bool acc = metropolis(unif(d.f3, FLIP), __fsub_rn(e_new, e_old), invT, T);
  r.n = acc ? nn : n;
  r.bond = acc ? b_new : b_old;
  r.single = acc ? s_new : s_old;
  r.rot = acc ? 1u : 0u;
  r.flip = 0u;
  if (FLIP) {
    const Vec3 f{-r.n.x, -r.n.y, -r.n.z};
    const float bf = bond_sum<POT>(m, f, nb, w), sf = single_energy(m, f, sid, s, elecE);
    const float e_cur = __fadd_rn(r.bond, r.single);
    if (metropolis(unif(d.f4, FLIP), __fsub_rn(__fadd_rn(bf, sf), e_cur), invT, T)) {
      r.n = f;
      r.bond = bf;
      r.single = sf;
      r.flip = 1u;
    }
  }
  return r;
}

// Energy of one site (all terms), for the observables of the untiled path.
template <int POT>
__device__ __forceinline__ float site_energy(const ModelDev &m, const Vec3 &x, const Vec3 (&nb)[6], const float (&w)[6],
                                             int sid, const Vec3 &s, float elecE) {
  return __fadd_rn(bond_sum<POT>(m, x, nb, w), single_energy(m, x, sid, s, elecE));
}

}  // namespace mcl
