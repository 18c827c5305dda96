// Site energies with the reference CPU's own float/double typing, for the reference-order replay kernel.
//
// Double literals and double bond accumulators are kept where src/potential.cpp, src/geometry.cpp and
// src/anchoring_*.cpp have them, and the translation unit that includes this header is compiled with
// -fmad=false, so every operation rounds exactly as the reference's x86-64 build (no FMA) does. Only the libm
// calls (sinf, cosf, expf) may differ from glibc by an ulp; the replay test reports the few decisions whose
// random number lies that close to the acceptance threshold.
#pragma once
#include "common.cuh"

namespace mcl {
namespace exact {

// src/potential.cpp:28-31
__device__ inline float ll(const ModelDev &m, const float ni[3], const float nj[3]) {
  float nij = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  return (float)((double)(-m.A) * 1.5 * (double)nij * (double)nij);
}

// src/potential.cpp:40-56
__device__ inline float ghrl(const ModelDev &m, const float ni[3], const float nj[3], const float r[3]) {
  float ai = ni[0] * r[0] + ni[1] * r[1] + ni[2] * r[2];
  float aj = nj[0] * r[0] + nj[1] * r[1] + nj[2] * r[2];
  float nij = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  float pij = 1.5f * nij * nij - 0.5f;
  float cross = (ni[2] * nj[1] - ni[1] * nj[2]) * r[0] + (ni[0] * nj[2] - ni[2] * nj[0]) * r[1] +
                (ni[1] * nj[0] - ni[0] * nj[1]) * r[2];
  float e1 = (float)((1.5 * (double)ai * (double)ai) + (1.5 * (double)aj * (double)aj) - 1);
  float t1 = e1 * (m.rho * pij + m.lam);
  float t2 = ai * aj * nij;
  double acc = (double)t1 + (double)m.mu * ((double)t2 - 1.0 / 9);
  acc = acc + (double)(m.nu * pij);
  float t4 = m.sigma * (float)(nij > 0 ? 1 : -1) * cross;
  acc = acc + (double)t4;
  return (float)acc;
}

// src/potential.cpp:19-24
__device__ inline float pear(const ModelDev &m, const float ni[3], const float nj[3], const float r[3]) {
  float nij = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  float ps = (1 + 2 * nij + nij * nij) * ((nj[0] - ni[0]) * r[0] + (nj[1] - ni[1]) * r[1] + (nj[2] - ni[2]) * r[2]);
  float f = -m.A * nij * nij - m.B1 * nij;
  return (float)((double)f - ((double)m.C * 0.25) * (double)ps);
}

template <int POT>
__device__ inline float pot(const ModelDev &m, const float ni[3], const float nj[3], const float r[3]) {
  if (POT == POT_GHRL) return ghrl(m, ni, nj, r);
  if (POT == POT_PEAR) return pear(m, ni, nj, r);
  return ll(m, ni, nj);
}

// src/potential.cpp:59-63
__device__ inline float field(const ModelDev &m, const float n[3], float elecE) {
  float ne = elecE * (n[0] * m.fdir[0] + n[1] * m.fdir[1] + n[2] * m.fdir[2]);
  return -m.elecP * ne - m.elecA * ne * ne;
}

// src/anchoring_{homeotropic,rp,rp_tangent,fg}.cpp (W included); the lab axis comes precomputed from the host.
__device__ inline float anchoring(const ModelDev &m, int sid, const float n[3], const float s[3]) {
  const float W = m.anch_W[sid];
  const float *lab = m.anch_lab[sid];
  float e[3], nij;
  switch (m.anch_type[sid]) {
    case ANCH_HOMEOTROPIC:
      nij = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
      return -W * nij * nij;
    case ANCH_RP:
      nij = n[0] * lab[0] + n[1] * lab[1] + n[2] * lab[2];
      return -W * nij * nij;
    case ANCH_RP_TANGENT: {
      float ds = lab[0] * s[0] + lab[1] * s[1] + lab[2] * s[2];
      e[0] = lab[0] - ds * s[0];
      e[1] = lab[1] - ds * s[1];
      e[2] = lab[2] - ds * s[2];
      float mod = sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
      if (mod < 1e-3f) return 0;
      e[0] /= mod;
      e[1] /= mod;
      e[2] /= mod;
      nij = n[0] * e[0] + n[1] * e[1] + n[2] * e[2];
      return -W * nij * nij;
    }
    case ANCH_FG:
      nij = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
      return +W * nij * nij;
    case ANCH_HOMEOTROPIC_GHRL:
      return W * ghrl(m, n, s, s);
    case ANCH_RP_GHRL:
      return W * ghrl(m, n, lab, s);
    case ANCH_FG_GHRL: {
      float ns = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
      float nj[3] = {n[0] - ns * s[0], n[1] - ns * s[1], n[2] - ns * s[2]};
      float mod = sqrtf(nj[0] * nj[0] + nj[1] * nj[1] + nj[2] * nj[2]);
      if (mod < 1e-6f) return 0;
      nj[0] /= mod;
      nj[1] /= mod;
      nj[2] /= mod;
      return W * ghrl(m, n, nj, s);
    }
  }
  return 0;
}

// src/geometry.cpp:23-76 (double accumulator) + site_energy of the geometries.
template <int POT>
__device__ inline float site_energy(const ModelDev &m, const float n[3], const float (&nb)[6][3], unsigned present,
                                    int sid, const float s[3], float elecE) {
  const float R[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  double E = 0;
#pragma unroll
  for (int d = 0; d < 6; d++)
    if (present & (1u << d)) E += pot<POT>(m, n, nb[d], R[d]);
  float Ef = (float)E;
  if (sid >= 0) Ef += anchoring(m, sid, n, s);
  if (m.field_on) Ef += field(m, n, elecE);
  return Ef;
}

}  // namespace exact
}  // namespace mcl
