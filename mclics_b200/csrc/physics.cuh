// Site energies for the production kernels: pair potentials, anchoring and field, FP32 with FMA.
//
// Definitions follow the reference CPU code (src/potential.cpp:19-63, src/anchoring_*.cpp,
// src/geometry*.cpp site_energy): E_site = sum over present neighbours of U(n, n_j, r_j) + [surface] anchoring
// + [elecA or elecP != 0] field. Neighbour order +x, -x, +y, -y, +z, -z (src/geometry.cpp:23-76); the bond vector
// r_j is a compile-time unit vector here, so its zero components cost nothing.
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
  float b = dot(x, y);
  return (-1.5f * m.A) * b * b;
}

// GHRL with bond vector r = sign * e_axis, src/potential.cpp:40-56.
template <int AXIS>
__device__ __forceinline__ float ghrl_bond(const ModelDev &m, const Vec3 &x, const Vec3 &y, float sign) {
  float ai = comp(x, AXIS), aj = comp(y, AXIS);  // a_i a_j and a^2 do not depend on the sign of r
  float b = dot(x, y);
  float p2 = fmaf(1.5f * b, b, -0.5f);
  float e1 = fmaf(1.5f, fmaf(ai, ai, aj * aj), -1.f);
  float u = fmaf(e1, fmaf(m.rho, p2, m.lam), fmaf(m.mu, fmaf(ai * aj, b, -1.f / 9.f), m.nu * p2));
  if (m.sigma != 0.f) {
    // c = r . (n_j x n_i)
    float c = AXIS == 0 ? (y.y * x.z - y.z * x.y) : (AXIS == 1 ? (y.z * x.x - y.x * x.z) : (y.x * x.y - y.y * x.x));
    u = fmaf(m.sigma * sign * (b > 0.f ? 1.f : -1.f), c, u);
  }
  return u;
}

// GHRL with an arbitrary bond vector (anchoring phantom neighbour along the surface normal).
__device__ __forceinline__ float ghrl_general(const ModelDev &m, const Vec3 &x, const Vec3 &y, const Vec3 &r) {
  float ai = dot(x, r), aj = dot(y, r), b = dot(x, y);
  float p2 = fmaf(1.5f * b, b, -0.5f);
  float e1 = fmaf(1.5f, fmaf(ai, ai, aj * aj), -1.f);
  float u = fmaf(e1, fmaf(m.rho, p2, m.lam), fmaf(m.mu, fmaf(ai * aj, b, -1.f / 9.f), m.nu * p2));
  if (m.sigma != 0.f) {
    float c = r.x * (y.y * x.z - y.z * x.y) + r.y * (y.z * x.x - y.x * x.z) + r.z * (y.x * x.y - y.y * x.x);
    u = fmaf(m.sigma * (b > 0.f ? 1.f : -1.f), c, u);
  }
  return u;
}

// Pear (Dhakal & Selinger), src/potential.cpp:19-24: -A b^2 - B1 b - C/4 (1+b)^2 r.(n_j - n_i).
template <int AXIS>
__device__ __forceinline__ float pear_bond(const ModelDev &m, const Vec3 &x, const Vec3 &y, float sign) {
  float b = dot(x, y);
  float opb = 1.f + b;
  float ps = opb * opb * (sign * (comp(y, AXIS) - comp(x, AXIS)));
  return fmaf(-m.A * b, b, fmaf(-m.B1, b, -0.25f * m.C * ps));
}

template <int POT, int D>
__device__ __forceinline__ float bond(const ModelDev &m, const Vec3 &x, const Vec3 &y) {
  if (POT == POT_LL) return ll_bond(m, x, y);
  if (POT == POT_GHRL) return ghrl_bond<BondDir<D>::axis>(m, x, y, BondDir<D>::sign);
  return pear_bond<BondDir<D>::axis>(m, x, y, BondDir<D>::sign);
}

// Sum over the six bonds; absent neighbours (free edge, empty site) are skipped.
template <int POT>
__device__ __forceinline__ float bond_sum(const ModelDev &m, const Vec3 &x, const Vec3 (&nb)[6], unsigned present) {
  float e = 0.f;
  if (present & 1u) e += bond<POT, 0>(m, x, nb[0]);
  if (present & 2u) e += bond<POT, 1>(m, x, nb[1]);
  if (present & 4u) e += bond<POT, 2>(m, x, nb[2]);
  if (present & 8u) e += bond<POT, 3>(m, x, nb[3]);
  if (present & 16u) e += bond<POT, 4>(m, x, nb[4]);
  if (present & 32u) e += bond<POT, 5>(m, x, nb[5]);
  return e;
}

// Field, src/potential.cpp:59-63.
__device__ __forceinline__ float field_energy(const ModelDev &m, const Vec3 &x, float elecE) {
  float ne = elecE * fmaf(x.x, m.fdir[0], fmaf(x.y, m.fdir[1], x.z * m.fdir[2]));
  return -m.elecP * ne - m.elecA * ne * ne;
}

// Anchoring of surface sid for a site with outward normal s (src/anchoring_*.cpp surface_potential, W included).
__device__ __forceinline__ float anchoring_energy(const ModelDev &m, int sid, const Vec3 &x, const Vec3 &s) {
  const float W = m.anch_W[sid];
  const Vec3 lab{m.anch_lab[sid][0], m.anch_lab[sid][1], m.anch_lab[sid][2]};
  switch (m.anch_type[sid]) {
    case ANCH_HOMEOTROPIC: {
      float c = dot(x, s);
      return -W * c * c;
    }
    case ANCH_RP: {
      float c = dot(x, lab);
      return -W * c * c;
    }
    case ANCH_RP_TANGENT: {
      float ds = dot(lab, s);
      Vec3 e{lab.x - ds * s.x, lab.y - ds * s.y, lab.z - ds * s.z};
      float mod = sqrtf(dot(e, e));
      if (mod < 1e-3f) return 0.f;
      float c = dot(x, e) / mod;
      return -W * c * c;
    }
    case ANCH_FG: {
      float c = dot(x, s);
      return W * c * c;
    }
    case ANCH_HOMEOTROPIC_GHRL:
      return W * ghrl_general(m, x, s, s);
    case ANCH_RP_GHRL:
      return W * ghrl_general(m, x, lab, s);
    case ANCH_FG_GHRL: {
      float c = dot(x, s);
      Vec3 t{x.x - c * s.x, x.y - c * s.y, x.z - c * s.z};
      float mod = sqrtf(dot(t, t));
      if (mod < 1e-6f) return 0.f;
      float inv = 1.f / mod;
      Vec3 tn{t.x * inv, t.y * inv, t.z * inv};
      return W * ghrl_general(m, x, tn, s);
    }
  }
  return 0.f;
}

// Full site energy. sid < 0 means not a surface site.
template <int POT>
__device__ __forceinline__ float site_energy(const ModelDev &m, const Vec3 &x, const Vec3 (&nb)[6], unsigned present,
                                             int sid, const Vec3 &s, float elecE) {
  float e = bond_sum<POT>(m, x, nb, present);
  if (sid >= 0) e += anchoring_energy(m, sid, x, s);
  if (m.field_on) e += field_energy(m, x, elecE);
  return e;
}

// Trial rotation by pi*va about the axis chosen by u2 (src/evolve.cpp:153-176), renormalised.
__device__ __forceinline__ Vec3 rotate_trial(const Vec3 &n, float va, int axis) {
  float s, c;
  sincospif(va, &s, &c);
  Vec3 r;
  if (axis == 0) {
    r = Vec3{n.x, fmaf(n.y, c, n.z * s), fmaf(n.z, c, -n.y * s)};
  } else if (axis == 1) {
    r = Vec3{fmaf(n.x, c, -n.z * s), n.y, fmaf(n.z, c, n.x * s)};
  } else {
    r = Vec3{fmaf(n.x, c, n.y * s), fmaf(n.y, c, -n.x * s), n.z};
  }
  float inv = rsqrtf(dot(r, r));
  return Vec3{r.x * inv, r.y * inv, r.z * inv};
}

// Metropolis test u < exp(-dE/T); T = 0 accepts when the energy does not increase (src/evolve.cpp:185-188).
__device__ __forceinline__ bool metropolis(float u, float dE, float invT, float T) {
  if (T > 0.f) return u < __expf(-dE * invT);
  return dE <= 0.f;
}

}  // namespace mcl
