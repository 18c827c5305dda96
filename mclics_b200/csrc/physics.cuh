// Site energies and the trial move for the production kernels, written once over a lane type L:
//   L = float   one site per thread (untiled kernels),
//   L = float2  two sites per thread, computed with Blackwell's paired FP32 instructions (FFMA2/FMUL2/FADD2:
//               __ffma2_rn, __fmul2_rn, __fadd2_rn), one site per lane.
// Every floating-point operation is explicit (fmaf / __fmul_rn / __fadd_rn or their paired forms), so both lane
// types round identically and the fused and untiled kernels take the same decisions.
//
// Definitions follow the reference CPU code (src/potential.cpp:19-63, src/anchoring_*.cpp,
// src/geometry*.cpp site_energy): E_site = sum over present neighbours of U(n, n_j, r_j) + [surface] anchoring
// + [elecA or elecP != 0] field. Neighbour order +x, -x, +y, -y, +z, -z (src/geometry.cpp:23-76); the bond vector
// r_j is a compile-time unit vector here, so its zero components cost nothing. An absent neighbour has weight 0.
#pragma once
#include "common.cuh"

namespace mcl {

// ---- lane operations ---------------------------------------------------------------------------------------
struct B2 {
  bool x, y;
};
template <typename L>
struct LaneBool;
template <>
struct LaneBool<float> {
  using type = bool;
};
template <>
struct LaneBool<float2> {
  using type = B2;
};
template <typename L>
using LB = typename LaneBool<L>::type;

__device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float2 fma_(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float mul_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float2 mul_(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float add_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 add_(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float neg_(float a) { return -a; }
__device__ __forceinline__ float2 neg_(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float sub_(float a, float b) { return __fadd_rn(a, -b); }
__device__ __forceinline__ float2 sub_(float2 a, float2 b) { return __fadd2_rn(a, neg_(b)); }
template <typename L>
__device__ __forceinline__ L splat(float v);
template <>
__device__ __forceinline__ float splat<float>(float v) { return v; }
template <>
__device__ __forceinline__ float2 splat<float2>(float v) { return make_float2(v, v); }
__device__ __forceinline__ float sel_(bool c, float a, float b) { return c ? a : b; }
__device__ __forceinline__ float2 sel_(B2 c, float2 a, float2 b) { return make_float2(c.x ? a.x : b.x, c.y ? a.y : b.y); }
__device__ __forceinline__ bool gt0(float a) { return a > 0.f; }
__device__ __forceinline__ B2 gt0(float2 a) { return B2{a.x > 0.f, a.y > 0.f}; }
__device__ __forceinline__ float sign_(float b) { return b > 0.f ? 1.f : -1.f; }
__device__ __forceinline__ float2 sign_(float2 b) { return make_float2(b.x > 0.f ? 1.f : -1.f, b.y > 0.f ? 1.f : -1.f); }

template <typename L>
struct V3 {
  L x, y, z;
};
using Vec3 = V3<float>;

template <typename L>
__device__ __forceinline__ L dot(const V3<L> &a, const V3<L> &b) {
  return fma_(a.x, b.x, fma_(a.y, b.y, mul_(a.z, b.z)));
}
template <int C, typename L>
__device__ __forceinline__ L comp(const V3<L> &a) {
  return C == 0 ? a.x : (C == 1 ? a.y : a.z);
}

// Bond D = 0..5 is +x, -x, +y, -y, +z, -z: axis D/2, sign +1 for even D.
template <int D>
struct BondDir {
  static constexpr int axis = D / 2;
  static constexpr float sign = (D % 2 == 0) ? 1.f : -1.f;
};

// Lebwohl-Lasher, src/potential.cpp:28-31: -1.5 A (n.n_j)^2.
template <typename L>
__device__ __forceinline__ L ll_bond(const ModelDev &m, const V3<L> &x, const V3<L> &y) {
  const L b = dot(x, y);
  return mul_(splat<L>(-1.5f * m.A), mul_(b, b));
}

// GHRL with bond vector r = sign * e_axis, src/potential.cpp:40-56. CHIRAL = false drops the sigma term, which
// is exact for sigma = 0 (fma(0, c, u) == u).
template <int AXIS, bool CHIRAL, typename L>
__device__ __forceinline__ L ghrl_bond(const ModelDev &m, const V3<L> &x, const V3<L> &y, float sign) {
  const L ai = comp<AXIS>(x), aj = comp<AXIS>(y);  // a_i a_j and a^2 do not depend on the sign of r
  const L b = dot(x, y);
  const L p2 = fma_(mul_(splat<L>(1.5f), b), b, splat<L>(-0.5f));
  const L e1 = fma_(splat<L>(1.5f), fma_(ai, ai, mul_(aj, aj)), splat<L>(-1.f));
  L u = fma_(e1, fma_(splat<L>(m.rho), p2, splat<L>(m.lam)),
             fma_(splat<L>(m.mu), fma_(mul_(ai, aj), b, splat<L>(-1.f / 9.f)), mul_(splat<L>(m.nu), p2)));
  if (CHIRAL) {
    // c = r . (n_j x n_i)
    const L c = AXIS == 0 ? fma_(y.y, x.z, neg_(mul_(y.z, x.y)))
                          : (AXIS == 1 ? fma_(y.z, x.x, neg_(mul_(y.x, x.z))) : fma_(y.x, x.y, neg_(mul_(y.y, x.x))));
    u = fma_(mul_(splat<L>(m.sigma * sign), sign_(b)), c, u);
  }
  return u;
}

// GHRL with an arbitrary bond vector (anchoring phantom neighbour along the surface normal), one site.
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
template <int AXIS, typename L>
__device__ __forceinline__ L pear_bond(const ModelDev &m, const V3<L> &x, const V3<L> &y, float sign) {
  const L b = dot(x, y);
  const L opb = add_(splat<L>(1.f), b);
  const L diff = sub_(comp<AXIS>(y), comp<AXIS>(x));
  const L ps = mul_(mul_(opb, opb), sign > 0.f ? diff : neg_(diff));
  return fma_(mul_(splat<L>(-m.A), b), b, fma_(splat<L>(-m.B1), b, mul_(splat<L>(-0.25f * m.C), ps)));
}

template <int POT, int D, bool CHIRAL, typename L>
__device__ __forceinline__ L bond(const ModelDev &m, const V3<L> &x, const V3<L> &y) {
  if (POT == POT_LL) return ll_bond(m, x, y);
  if (POT == POT_GHRL) return ghrl_bond<BondDir<D>::axis, CHIRAL>(m, x, y, BondDir<D>::sign);
  return pear_bond<BondDir<D>::axis>(m, x, y, BondDir<D>::sign);
}

// Bond sums of one or two directors over the six bonds, with weights w[d] in {0, 1} (0: free edge or empty
// site). PXY = true: the x and y neighbours are known to be present, their weights are not applied (exact: the
// weight would be 1). The two-director form evaluates both in one pass, so each neighbour is used once.
template <int POT, bool PXY, bool CHIRAL, int D, typename L>
__device__ __forceinline__ L acc_bond(const ModelDev &m, const V3<L> &x, const V3<L> &y, const L &w, const L &e) {
  const L u = bond<POT, D, CHIRAL>(m, x, y);
  if (PXY && D < 4) return D == 0 ? u : add_(e, u);
  return D == 0 ? mul_(w, u) : fma_(w, u, e);
}

// Lebwohl-Lasher sums: sum_j w_j (n.n_j)^2 over the six bonds, then one multiplication by -1.5 A (the bond
// energy is that constant times a square, so it factors out of the sum).
template <bool PXY, int D, typename L>
__device__ __forceinline__ L ll_acc(const V3<L> &x, const V3<L> &y, const L &w, const L &s) {
  const L b = dot(x, y);
  if (PXY && D < 4) return D == 0 ? mul_(b, b) : fma_(b, b, s);
  return D == 0 ? mul_(mul_(w, b), b) : fma_(mul_(w, b), b, s);
}
template <bool PXY, typename L>
__device__ __forceinline__ L ll_sum(const ModelDev &m, const V3<L> &x, const V3<L> (&nb)[6], const L (&w)[6]) {
  L s = ll_acc<PXY, 0>(x, nb[0], w[0], w[0]);
  s = ll_acc<PXY, 1>(x, nb[1], w[1], s);
  s = ll_acc<PXY, 2>(x, nb[2], w[2], s);
  s = ll_acc<PXY, 3>(x, nb[3], w[3], s);
  s = ll_acc<PXY, 4>(x, nb[4], w[4], s);
  s = ll_acc<PXY, 5>(x, nb[5], w[5], s);
  return mul_(splat<L>(-1.5f * m.A), s);
}

// GHRL without the chiral term as sums over the site's bonds. With a_i = n.r, a_j = n_j.r, b = n.n_j, the pair
// energy of ghrl_bond is
//   U = (1.5 a_i^2 + K) P + mu a_i a_j b + 1.5 nu b^2 + c0,   K = 1.5 a_j^2 - 1,   P = 1.5 rho b^2 + lambda - rho / 2,
//   c0 = -mu / 9 - nu / 2,
// so the site sums to sum_d [(A_a(d) + K_d) P_d + 1.5 nu B_d] + mu sum_a a_i,a (sum_{d on a} a_j,d b_d) + c0 sum_d w_d
// (A_a = 1.5 a_i,a^2, B = b^2; an absent bond has w = 0, applied by scaling b and A + K). NS directors (1: one
// site energy; 2: the old and new director of a trial) go through the bonds together, so each neighbour and its
// K_d are used by both and then released.
template <bool PXY, int NS, typename L>
__device__ __forceinline__ void ghrl_sums(const ModelDev &m, const V3<L> *const (&x)[NS], const V3<L> (&nb)[6],
                                          const L (&w)[6], L (&out)[NS]) {
  const L h3 = splat<L>(1.5f), r15 = splat<L>(1.5f * m.rho), lamp = splat<L>(fmaf(-0.5f, m.rho, m.lam));
  L e[NS], sB[NS];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    L A[NS], mab[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
      const L ai = a == 0 ? x[i]->x : (a == 1 ? x[i]->y : x[i]->z);
      A[i] = mul_(mul_(h3, ai), ai);
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int d = 2 * a + s;
      const L aj = a == 0 ? nb[d].x : (a == 1 ? nb[d].y : nb[d].z);
      const L K = fma_(mul_(h3, aj), aj, splat<L>(-1.f));
#pragma unroll
      for (int i = 0; i < NS; i++) {
        L b = dot(*x[i], nb[d]), t = add_(A[i], K);
        if (!(PXY && d < 4)) {
          b = mul_(w[d], b);
          t = mul_(w[d], t);
        }
        const L B = mul_(b, b), P = fma_(r15, B, lamp);
        e[i] = d == 0 ? mul_(t, P) : fma_(t, P, e[i]);
        sB[i] = d == 0 ? B : add_(sB[i], B);
        mab[i] = s == 0 ? mul_(aj, b) : fma_(aj, b, mab[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < NS; i++) {
      const L ai = a == 0 ? x[i]->x : (a == 1 ? x[i]->y : x[i]->z);
      e[i] = fma_(mul_(splat<L>(m.mu), ai), mab[i], e[i]);
    }
  }
  const L nw = PXY ? add_(add_(w[4], w[5]), splat<L>(4.f))
                   : add_(add_(add_(w[0], w[1]), add_(w[2], w[3])), add_(w[4], w[5]));
  const L c = mul_(splat<L>(m.ghrl_c0), nw);
#pragma unroll
  for (int i = 0; i < NS; i++) out[i] = fma_(splat<L>(1.5f * m.nu), sB[i], add_(e[i], c));
}

template <int POT, bool PXY, bool CHIRAL, typename L>
__device__ __forceinline__ L bond_sum(const ModelDev &m, const V3<L> &x, const V3<L> (&nb)[6], const L (&w)[6]) {
  if (POT == POT_LL) return ll_sum<PXY>(m, x, nb, w);
  if (POT == POT_GHRL && !CHIRAL) {
    const V3<L> *const xs[1] = {&x};
    L out[1];
    ghrl_sums<PXY, 1>(m, xs, nb, w, out);
    return out[0];
  }
  L e = acc_bond<POT, PXY, CHIRAL, 0>(m, x, nb[0], w[0], w[0]);
  e = acc_bond<POT, PXY, CHIRAL, 1>(m, x, nb[1], w[1], e);
  e = acc_bond<POT, PXY, CHIRAL, 2>(m, x, nb[2], w[2], e);
  e = acc_bond<POT, PXY, CHIRAL, 3>(m, x, nb[3], w[3], e);
  e = acc_bond<POT, PXY, CHIRAL, 4>(m, x, nb[4], w[4], e);
  e = acc_bond<POT, PXY, CHIRAL, 5>(m, x, nb[5], w[5], e);
  return e;
}

template <int POT, bool PXY, bool CHIRAL, typename L>
__device__ __forceinline__ void bond_sum2(const ModelDev &m, const V3<L> &x, const V3<L> &x2, const V3<L> (&nb)[6],
                                          const L (&w)[6], L &e1, L &e2) {
  if (POT == POT_LL) {
    L s1 = ll_acc<PXY, 0>(x, nb[0], w[0], w[0]), s2 = ll_acc<PXY, 0>(x2, nb[0], w[0], w[0]);
    s1 = ll_acc<PXY, 1>(x, nb[1], w[1], s1);
    s2 = ll_acc<PXY, 1>(x2, nb[1], w[1], s2);
    s1 = ll_acc<PXY, 2>(x, nb[2], w[2], s1);
    s2 = ll_acc<PXY, 2>(x2, nb[2], w[2], s2);
    s1 = ll_acc<PXY, 3>(x, nb[3], w[3], s1);
    s2 = ll_acc<PXY, 3>(x2, nb[3], w[3], s2);
    s1 = ll_acc<PXY, 4>(x, nb[4], w[4], s1);
    s2 = ll_acc<PXY, 4>(x2, nb[4], w[4], s2);
    s1 = ll_acc<PXY, 5>(x, nb[5], w[5], s1);
    s2 = ll_acc<PXY, 5>(x2, nb[5], w[5], s2);
    e1 = mul_(splat<L>(-1.5f * m.A), s1);
    e2 = mul_(splat<L>(-1.5f * m.A), s2);
    return;
  }
  if (POT == POT_GHRL && !CHIRAL) {
    const V3<L> *const xs[2] = {&x, &x2};
    L out[2];
    ghrl_sums<PXY, 2>(m, xs, nb, w, out);
    e1 = out[0];
    e2 = out[1];
    return;
  }
  e1 = acc_bond<POT, PXY, CHIRAL, 0>(m, x, nb[0], w[0], w[0]);
  e2 = acc_bond<POT, PXY, CHIRAL, 0>(m, x2, nb[0], w[0], w[0]);
  e1 = acc_bond<POT, PXY, CHIRAL, 1>(m, x, nb[1], w[1], e1);
  e2 = acc_bond<POT, PXY, CHIRAL, 1>(m, x2, nb[1], w[1], e2);
  e1 = acc_bond<POT, PXY, CHIRAL, 2>(m, x, nb[2], w[2], e1);
  e2 = acc_bond<POT, PXY, CHIRAL, 2>(m, x2, nb[2], w[2], e2);
  e1 = acc_bond<POT, PXY, CHIRAL, 3>(m, x, nb[3], w[3], e1);
  e2 = acc_bond<POT, PXY, CHIRAL, 3>(m, x2, nb[3], w[3], e2);
  e1 = acc_bond<POT, PXY, CHIRAL, 4>(m, x, nb[4], w[4], e1);
  e2 = acc_bond<POT, PXY, CHIRAL, 4>(m, x2, nb[4], w[4], e2);
  e1 = acc_bond<POT, PXY, CHIRAL, 5>(m, x, nb[5], w[5], e1);
  e2 = acc_bond<POT, PXY, CHIRAL, 5>(m, x2, nb[5], w[5], e2);
}

// Field, src/potential.cpp:59-63.
template <typename L>
__device__ __forceinline__ L field_energy(const ModelDev &m, const V3<L> &x, float elecE) {
  const L ne = mul_(splat<L>(elecE),
                    fma_(x.x, splat<L>(m.fdir[0]), fma_(x.y, splat<L>(m.fdir[1]), mul_(x.z, splat<L>(m.fdir[2])))));
  return fma_(splat<L>(-m.elecA), mul_(ne, ne), mul_(splat<L>(-m.elecP), ne));
}

// Anchoring of one surface for a site with outward normal s (src/anchoring_*.cpp surface_potential, W included).
// Not inlined: surface sites are rare, and the seven anchoring forms would otherwise claim registers in every
// sweep kernel's hot loop. Arguments by value (a reference to the kernel's model parameter would force a copy).
static __device__ __noinline__ float anchoring_core(int type, float W, float lx, float ly, float lz, float lam, float mu,
                                                    float nu, float rho, float sigma, float x0, float x1, float x2,
                                                    float s0, float s1, float s2) {
  ModelDev m;  // only the GHRL coefficients are read below
  m.lam = lam;
  m.mu = mu;
  m.nu = nu;
  m.rho = rho;
  m.sigma = sigma;
  const Vec3 x{x0, x1, x2}, s{s0, s1, s2}, lab{lx, ly, lz};
  switch (type) {
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

__device__ __forceinline__ float anchoring_energy(const ModelDev &m, int sid, const Vec3 &x, const Vec3 &s) {
  return anchoring_core(m.anch_type[sid], m.anch_W[sid], m.anch_lab[sid][0], m.anch_lab[sid][1], m.anch_lab[sid][2],
                        m.lam, m.mu, m.nu, m.rho, m.sigma, x.x, x.y, x.z, s.x, s.y, s.z);
}

// Single-site terms: anchoring (sid >= 0, the same surface for both lanes) and, with FIELD, the field (FIELD is
// false only when elecA = elecP = 0, where the reference adds no field term either).
template <bool FIELD>
__device__ __forceinline__ float single_energy(const ModelDev &m, const Vec3 &x, int sid, const Vec3 &s, float elecE) {
  float e = 0.f;
  if (sid >= 0) e = anchoring_energy(m, sid, x, s);
  if (FIELD && m.field_on) e = __fadd_rn(e, field_energy(m, x, elecE));
  return e;
}
template <bool FIELD>
__device__ __forceinline__ float2 single_energy(const ModelDev &m, const V3<float2> &x, int sid, const Vec3 &s,
                                                float elecE) {
  float2 e = make_float2(0.f, 0.f);
  if (sid >= 0) {
    e.x = anchoring_energy(m, sid, Vec3{x.x.x, x.y.x, x.z.x}, s);
    e.y = anchoring_energy(m, sid, Vec3{x.x.y, x.y.y, x.z.y}, s);
  }
  if (FIELD && m.field_on) e = __fadd2_rn(e, field_energy(m, x, elecE));
  return e;
}

// Per-lane transcendental helpers.
__device__ __forceinline__ void sincos_pi(float va, float &s, float &c) { __sincosf(__fmul_rn(3.14159265358979f, va), &s, &c); }
__device__ __forceinline__ void sincos_pi(float2 va, float2 &s, float2 &c) {
  sincos_pi(va.x, s.x, c.x);
  sincos_pi(va.y, s.y, c.y);
}
__device__ __forceinline__ float rsqrt_(float a) { return rsqrtf(a); }
__device__ __forceinline__ float2 rsqrt_(float2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }

// Trial rotation by pi * va about axis `axis` (src/evolve.cpp:153-176): the reference's three rotations in one
// branch-free Rodrigues form n' = c n + (1 - c) n_a e_a - s (e_a x n), then renormalised. w0..w2: one-hot axis.
template <typename L>
__device__ __forceinline__ V3<L> rotate_trial(const V3<L> &n, L va, L w0, L w1, L w2) {
  L s, c;
  sincos_pi(va, s, c);  // |pi va| <= pi: the hardware sin/cos range
  const L cx = fma_(w1, n.z, neg_(mul_(w2, n.y))), cy = fma_(w2, n.x, neg_(mul_(w0, n.z))),
          cz = fma_(w0, n.y, neg_(mul_(w1, n.x)));
  const L omc = sub_(splat<L>(1.f), c);
  const V3<L> r{fma_(c, n.x, fma_(mul_(omc, w0), n.x, neg_(mul_(s, cx)))),
                fma_(c, n.y, fma_(mul_(omc, w1), n.y, neg_(mul_(s, cy)))),
                fma_(c, n.z, fma_(mul_(omc, w2), n.z, neg_(mul_(s, cz))))};
  const L inv = rsqrt_(dot(r, r));
  return V3<L>{mul_(r.x, inv), mul_(r.y, inv), mul_(r.z, inv)};
}

// Metropolis test u < exp(-dE/T); T = 0 accepts when the energy does not increase (src/evolve.cpp:185-188).
__device__ __forceinline__ bool metropolis(float u, float dE, float invT, float T) {
  return T > 0.f ? (u < __expf(-__fmul_rn(dE, invT))) : (dE <= 0.f);
}
__device__ __forceinline__ B2 metropolis(float2 u, float2 dE, float invT, float T) {
  return B2{metropolis(u.x, dE.x, invT, T), metropolis(u.y, dE.y, invT, T)};
}

// Draw fields -> lane values.
template <typename L>
struct LaneDraw {
  L u1, u3, u4;   // angle, rotation acceptance, flip acceptance uniforms
  L w0, w1, w2;   // one-hot rotation axis
};
__device__ __forceinline__ LaneDraw<float> lane_draw(const Draw &d, bool flip) {
  LaneDraw<float> r;
  r.u1 = unif(d.f1, flip);
  r.u3 = unif(d.f3, flip);
  r.u4 = unif(d.f4, flip);
  const int a = rotation_axis(d.f2, flip);
  r.w0 = a == 0 ? 1.f : 0.f;
  r.w1 = a == 1 ? 1.f : 0.f;
  r.w2 = a == 2 ? 1.f : 0.f;
  return r;
}
__device__ __forceinline__ LaneDraw<float2> lane_draw(const Draw &d0, const Draw &d1, bool flip) {
  const LaneDraw<float> a = lane_draw(d0, flip), b = lane_draw(d1, flip);
  return LaneDraw<float2>{make_float2(a.u1, b.u1), make_float2(a.u3, b.u3), make_float2(a.u4, b.u4),
                          make_float2(a.w0, b.w0), make_float2(a.w1, b.w1), make_float2(a.w2, b.w2)};
}

// Result of one trial move per lane.
template <typename L>
struct SiteResultT {
  V3<L> n;       // director after the move
  L bond;        // bond energy of the final director
  L single;      // single-site energy of the final director
  LB<L> rot;     // rotation accepted
  LB<L> flip;    // flip accepted
};

template <typename L>
__device__ __forceinline__ V3<L> sel3(LB<L> c, const V3<L> &a, const V3<L> &b) {
  return V3<L>{sel_(c, a.x, b.x), sel_(c, a.y, b.y), sel_(c, a.z, b.z)};
}

// One trial move (src/evolve.cpp:133-207): rotation, Metropolis, then the optional n -> -n trial.
// Compile-time features: FLIP (n -> -n trial), PXY (x, y neighbours always present), CHIRAL (GHRL sigma term),
// FIELD (field term), SINGLE = false (the caller knows the site has no single-site term: no surface, no field;
// the energies are then the bond sums themselves, which is what adding the zero single term gives, up to the sign
// of a zero). Every combination rounds like the general one on the inputs it applies to.
template <int POT, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, typename L, bool SINGLE = true>
__device__ __forceinline__ SiteResultT<L> site_update(const ModelDev &m, const V3<L> &n, const V3<L> (&nb)[6],
                                                      const L (&w)[6], int sid, const Vec3 &s, float elecE,
                                                      const LaneDraw<L> &d, float av, float T, float invT) {
  const L va = mul_(fma_(splat<L>(2.f), d.u1, splat<L>(-1.f)), splat<L>(av));
  const V3<L> nn = rotate_trial(n, va, d.w0, d.w1, d.w2);
  L b_old, b_new;
  bond_sum2<POT, PXY, CHIRAL>(m, n, nn, nb, w, b_old, b_new);
  const L s_old = SINGLE ? single_energy<FIELD>(m, n, sid, s, elecE) : splat<L>(0.f);
  const L s_new = SINGLE ? single_energy<FIELD>(m, nn, sid, s, elecE) : splat<L>(0.f);
  const L e_old = SINGLE ? add_(b_old, s_old) : b_old, e_new = SINGLE ? add_(b_new, s_new) : b_new;
  SiteResultT<L> r;
  r.rot = metropolis(d.u3, sub_(e_new, e_old), invT, T);
  r.n = sel3<L>(r.rot, nn, n);
  r.bond = sel_(r.rot, b_new, b_old);
  r.single = SINGLE ? sel_(r.rot, s_new, s_old) : splat<L>(0.f);
  if (FLIP) {
    const V3<L> f{neg_(r.n.x), neg_(r.n.y), neg_(r.n.z)};
    const L bf = bond_sum<POT, PXY, CHIRAL>(m, f, nb, w);
    const L sf = SINGLE ? single_energy<FIELD>(m, f, sid, s, elecE) : splat<L>(0.f);
    const L e_cur = SINGLE ? add_(r.bond, r.single) : r.bond;
    r.flip = metropolis(d.u4, SINGLE ? sub_(add_(bf, sf), e_cur) : sub_(bf, e_cur), invT, T);
    r.n = sel3<L>(r.flip, f, r.n);
    r.bond = sel_(r.flip, bf, r.bond);
    r.single = sel_(r.flip, sf, r.single);
  } else {
    r.flip = LB<L>{};
  }
  return r;
}

// Energy of one site (all terms), for the observables of the untiled path.
template <int POT>
__device__ __forceinline__ float site_energy(const ModelDev &m, const Vec3 &x, const Vec3 (&nb)[6], const float (&w)[6],
                                             int sid, const Vec3 &s, float elecE) {
  return __fadd_rn(bond_sum<POT, false, true>(m, x, nb, w), single_energy<true>(m, x, sid, s, elecE));
}

}  // namespace mcl
