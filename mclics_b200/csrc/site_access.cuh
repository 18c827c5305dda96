// Gathering a site's environment from the padded SoA director buffers (simple kernels): its director, the six
// neighbours with their presence mask, and its surface id and normal.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace mcl {

__device__ __forceinline__ float ld_dir(const float *__restrict__ d, const RepDesc &R, int c, int x, int y, int z) {
  return __ldg(d + dir_index(R, c, x, y, z));
}

// Neighbour coordinate along one axis: periodic wraps, free marks -1 and N as absent
// (src/potential.cpp:64-74).
__device__ __forceinline__ bool nb_coord(int periodic, int v, int N, int &out) {
  if (periodic) {
    out = v < 0 ? v + N : (v >= N ? v - N : v);
    return true;
  }
  out = v;
  return v >= 0 && v < N;
}

__device__ __forceinline__ long long site_linear(const RepDesc &R, int x, int y, int z) {
  return (long long)x + (long long)R.nx * ((long long)y + (long long)R.ny * z);
}

// Surface of a slab site: surface 1 (normal +z) at z = nz-1, surface 0 (normal -z) at z = 0
// (src/geometry_slab.cpp:51-71; for nz = 1 the single plane is surface 1, as the reference overwrites it).
__device__ __forceinline__ int slab_surface(int z, int nz, float &sz) {
  if (z == nz - 1) {
    sz = 1.f;
    return 1;
  }
  if (z == 0) {
    sz = -1.f;
    return 0;
  }
  sz = 0.f;
  return -1;
}

// Returns false for an empty site. nb/present follow the bond order +x, -x, +y, -y, +z, -z.
template <int GEO>
__device__ __forceinline__ bool gather_site(const RepDesc &R, const float *__restrict__ dir,
                                            const uint8_t *__restrict__ pt, const float *__restrict__ nrm, int x, int y,
                                            int z, Vec3 &n, Vec3 (&nb)[6], unsigned &present, int &sid, Vec3 &s);

// The same with bond weights (1 present, 0 absent) instead of a bit mask.
template <int GEO>
__device__ __forceinline__ bool gather_site_w(const RepDesc &R, const float *__restrict__ dir,
                                              const uint8_t *__restrict__ pt, const float *__restrict__ nrm, int x,
                                              int y, int z, Vec3 &n, Vec3 (&nb)[6], float (&w)[6], int &sid, Vec3 &s) {
  unsigned present;
  if (!gather_site<GEO>(R, dir, pt, nrm, x, y, z, n, nb, present, sid, s)) return false;
#pragma unroll
  for (int d = 0; d < 6; d++) w[d] = (present >> d) & 1u ? 1.f : 0.f;
  return true;
}

template <int GEO>
__device__ __forceinline__ bool gather_site(const RepDesc &R, const float *__restrict__ dir,
                                            const uint8_t *__restrict__ pt, const float *__restrict__ nrm, int x, int y,
                                            int z, Vec3 &n, Vec3 (&nb)[6], unsigned &present, int &sid, Vec3 &s) {
  const long long site = site_linear(R, x, y, z);
  int p = 1;
  if (GEO == GEO_PT) {
    p = pt[R.site_off + site];
    if (p == 0) return false;
  }
  n = Vec3{ld_dir(dir, R, 0, x, y, z), ld_dir(dir, R, 1, x, y, z), ld_dir(dir, R, 2, x, y, z)};
  present = 0;
#pragma unroll
  for (int d = 0; d < 6; d++) {
    const int axis = d >> 1;
    const int delta = (d & 1) ? -1 : 1;
    int xx = x, yy = y, zz = z;
    bool ok;
    if (axis == 0)
      ok = nb_coord(R.periodic[0], x + delta, R.nx, xx);
    else if (axis == 1)
      ok = nb_coord(R.periodic[1], y + delta, R.ny, yy);
    else
      ok = nb_coord(R.periodic[2], z + delta, R.nz, zz);
    if (ok && GEO == GEO_PT) ok = pt[R.site_off + site_linear(R, xx, yy, zz)] != 0;
    if (ok) {
      nb[d] = Vec3{ld_dir(dir, R, 0, xx, yy, zz), ld_dir(dir, R, 1, xx, yy, zz), ld_dir(dir, R, 2, xx, yy, zz)};
      present |= 1u << d;
    } else {
      nb[d] = Vec3{0.f, 0.f, 0.f};
    }
  }
  sid = -1;
  s = Vec3{0.f, 0.f, 0.f};
  if (GEO == GEO_SLAB) {
    float sz;
    sid = slab_surface(z, R.nz, sz);
    s.z = sz;
  } else if (GEO == GEO_PT) {
    if (p >= 2) {
      sid = p - 2;
      const float *v = nrm + 3 * (R.site_off + site);
      s = Vec3{v[0], v[1], v[2]};
    }
  }
  return true;
}

// The same result as gather_site_w with less index arithmetic: one 64-bit base per row (y, z) of component 0, the
// other components at +comp and +2 comp, and x as (parity, half-row cell) within the row.
template <int GEO>
__device__ __forceinline__ bool gather_site_rows(const RepDesc &R, const float *__restrict__ dir,
                                                 const uint8_t *__restrict__ pt, const float *__restrict__ nrm, int x,
                                                 int y, int z, Vec3 &n, Vec3 (&nb)[6], float (&w)[6], int &sid,
                                                 Vec3 &s) {
  const long long site = site_linear(R, x, y, z);
  int p = 1;
  if (GEO == GEO_PT) {
    p = pt[R.site_off + site];
    if (p == 0) return false;
  }
  const long long comp = R.comp;
  auto row = [&](int yy, int zz) -> const float * {
    return dir + R.off + ((long long)zz * R.py + (yy + GY)) * R.px + GH;
  };
  auto cell = [&](int xx) -> int { return (xx & 1) * R.hp + (xx >> 1); };
  auto load = [&](const float *q) -> Vec3 { return Vec3{__ldg(q), __ldg(q + comp), __ldg(q + 2 * comp)}; };
  const float *r0 = row(y, z);
  const int c0 = cell(x);
  n = load(r0 + c0);
#pragma unroll
  for (int d = 0; d < 6; d++) {
    const int axis = d >> 1;
    const int delta = (d & 1) ? -1 : 1;
    int v;
    bool ok;
    const float *q;
    if (axis == 0) {
      ok = nb_coord(R.periodic[0], x + delta, R.nx, v);
      q = r0 + cell(v);
    } else if (axis == 1) {
      ok = nb_coord(R.periodic[1], y + delta, R.ny, v);
      q = row(v, z) + c0;
    } else {
      ok = nb_coord(R.periodic[2], z + delta, R.nz, v);
      q = row(y, v) + c0;
    }
    if (ok && GEO == GEO_PT) {
      const int xx = axis == 0 ? v : x, yy = axis == 1 ? v : y, zz = axis == 2 ? v : z;
      ok = pt[R.site_off + site_linear(R, xx, yy, zz)] != 0;
    }
    if (ok) {  // an absent neighbour's row may lie outside the replica (free z): never load it
      nb[d] = load(q);
      w[d] = 1.f;
    } else {
      nb[d] = Vec3{0.f, 0.f, 0.f};
      w[d] = 0.f;
    }
  }
  sid = -1;
  s = Vec3{0.f, 0.f, 0.f};
  if (GEO == GEO_SLAB) {
    float sz;
    sid = slab_surface(z, R.nz, sz);
    s.z = sz;
  } else if (GEO == GEO_PT) {
    if (p >= 2) {
      sid = p - 2;
      const float *v = nrm + 3 * (R.site_off + site);
      s = Vec3{v[0], v[1], v[2]};
    }
  }
  return true;
}

}  // namespace mcl
