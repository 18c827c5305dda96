// Shared device-side definitions: lattice layout, replica descriptors, model constants and the counter-based RNG.
//
// Director storage in HBM (per replica, per buffer): three FP32 component volumes (SoA). Every row of a plane is
// stored split by x parity: the even-x sites first, then the odd-x sites, each half-row padded by GH = 4 cells on
// the left and at least 4 on the right:
//   dir[off + (c * nz + z) * py * px + (y + GY) * px + (x & 1) * hp + (x >> 1) + GH],
// hp = round_up(ceil(nx / 2), 4) + 8, px = 2 hp, py = ny + 2 GY, GY = 2. One colour of the checkerboard in a row is
// thus one contiguous half-row, and a 16-byte aligned TMA box can start 4 cells left of any tile that begins at a
// multiple of 8 in x. For a periodic axis the cells x = -2, -1, nx, nx + 1 (likewise y) hold copies of the
// wrapped sites ("ghosts"); the fused kernel reads them instead of wrapping. Padding beyond is zero.
#pragma once
#include <math.h>
#include <stdint.h>

namespace mcl {

constexpr int GH = 4;  // left padding of a half-row
constexpr int GY = 2;
constexpr int kMaxSurfaces = 16;

enum Pot { POT_LL = 0, POT_GHRL = 1, POT_PEAR = 2 };
enum Geo { GEO_BULK = 0, GEO_SLAB = 1, GEO_PT = 2 };  // GEO_PT: sphere and custom (point types from memory)
enum Anch {
  ANCH_HOMEOTROPIC = 0,
  ANCH_RP = 1,
  ANCH_RP_TANGENT = 2,
  ANCH_FG = 3,
  ANCH_HOMEOTROPIC_GHRL = 4,
  ANCH_RP_GHRL = 5,
  ANCH_FG_GHRL = 6
};

// Model constants, passed by value to every kernel.
struct ModelDev {
  int potential;
  float A, B1, C;
  float lam, mu, nu, rho, sigma;  // GHRL
  float ghrl_c0;                  // -mu / 9 - nu / 2 (the constant of every GHRL bond), fmaf(-0.5f, nu, -mu / 9.f)
  float fdir[3];
  float elecA, elecP;
  int flip;
  int field_on;  // elecA != 0 || elecP != 0 (the reference adds the field term only then)
  int n_surf;
  int anch_type[kMaxSurfaces];
  float anch_W[kMaxSurfaces];
  float anch_lab[kMaxSurfaces][3];  // lab easy axis, computed on the host like anchoring.cpp:19-24
};

// Immutable per-replica layout.
struct RepDesc {
  int nx, ny, nz;
  int px, py;        // row pitch (2 hp) and padded rows per plane
  int geo;           // Geo
  int periodic[3];
  int hp;            // half-row pitch
  long long off;     // float offset of this replica in the director buffers
  long long comp;    // floats per component = nz * py * px
  long long site_off;  // offset of this replica in the unpadded per-site arrays (pt, normals, decisions)
  unsigned long long seed;
  double n_valid;
  // z-slab of a larger lattice (mcl_zslab_init): local planes 0 and nz - 1 are halo copies of the neighbours'
  // boundary planes, planes 1 .. nz - 2 are owned; local plane p is global plane zoff + p of a lattice of nzg
  // planes. Otherwise zslab = 0, zoff = 0, nzg = nz.
  int zslab, zoff, nzg;
};

// Mutable per-replica state (device memory).
struct RepState {
  float T, elecE, ang_var;
  float pad;  // acceptance fraction of the last sweep
  unsigned long long acc;  // accepted rotations in the current sweep
};

// One observables record (device memory, copied to mcl_observables on the host).
struct ObsRecord {
  double energy, q[6], S, director[3], nsum[3], n_valid, acceptance, ang_var, sweep;
};
// Per-block partial sums of the observables: energy, q[6], nsum[3].
constexpr int kPartials = 10;
// Per-replica sums a z-slab process contributes to the reduction over processes: the kPartials observables and
// the accepted rotations.
constexpr int kZslabSums = kPartials + 1;

__host__ __device__ inline long long dir_index(const RepDesc &r, int c, int x, int y, int z) {
  return r.off + (long long)c * r.comp + ((long long)z * r.py + (y + GY)) * r.px + (x & 1) * r.hp + (x >> 1) + GH;
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ------------------------------------------------------
// Every draw of this library uses a key fixed at compile time per stream and carries the seed in the counter:
// counter (a, b, seed_lo, seed_hi + c_hi), key (kPhiloxKey0 + stream, kPhiloxKey1). Philox under one key is a
// bijection of the 128-bit counter, so distinct (a, b, seed) give independent-looking blocks, and the ten round
// keys are constants the compiler folds into the XORs (no per-call key schedule). Site draws use a = site,
// b = sweep (low 32 bits), c_hi = sweep >> 32: two (seed, sweep) pairs share a counter only if their seeds differ
// in the upper 32 bits by minus the difference of their sweep counts' upper 32 bits. Streams: 0 plain move
// (u1 angle, u2 axis, u3 rotation accept, u4 flip accept), 1 learned proposal, 2 initial conditions, 3 training
// samples.
struct U4 {
  uint32_t x, y, z, w;
};

constexpr uint32_t kPhiloxKey0 = 0x694C634Du, kPhiloxKey1 = 0x30303242u;

__host__ __device__ __forceinline__ U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                      uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;  // one 32 x 32 -> 64 each
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return U4{c0, c1, c2, c3};
}

// One block of stream `stream` (a compile-time constant at every call site) at counter (a, b, seed, c_hi).
__host__ __device__ __forceinline__ U4 stream_draws(uint32_t a, uint32_t b, unsigned long long seed, uint32_t c_hi,
                                                     uint32_t stream) {
  return philox4x32_10(a, b, (uint32_t)seed, (uint32_t)(seed >> 32) + c_hi, kPhiloxKey0 + stream, kPhiloxKey1);
}

__host__ __device__ __forceinline__ U4 site_draws(unsigned long long seed, unsigned long long sweep, uint32_t site,
                                                   uint32_t stream) {
  return stream_draws(site, (uint32_t)sweep, seed, (uint32_t)(sweep >> 32), stream);
}

// ---- draws of one site -----------------------------------------------------------------------------------
// Flip models (pear, or a dipolar field): one Philox call per site, counter (site, sweep, 0), four 24-bit fields.
// Other models: one call per pair of same-colour sites x and x ^ 2 of a row, counter (linear index of
// (x & ~2, y, z), sweep, 0); the site takes the 64-bit half h = (x >> 1) & 1 and splits it into three 21-bit
// fields. Uniform = field * 2^-bits, exact in float and double.
struct Draw {
  uint32_t f1, f2, f3, f4;  // angle, axis, rotation acceptance, flip acceptance
};

__host__ __device__ __forceinline__ uint32_t pair_counter(uint32_t x, uint32_t y, uint32_t z, uint32_t nx, uint32_t ny) {
  return (x & ~2u) + nx * (y + ny * z);
}

__host__ __device__ __forceinline__ Draw pair_half(const U4 &o, uint32_t h) {
  const uint32_t lo = h ? o.z : o.x, hi = h ? o.w : o.y;
  Draw d;
  d.f1 = lo & 0x1FFFFFu;
  d.f2 = ((lo >> 21) | (hi << 11)) & 0x1FFFFFu;
  d.f3 = (hi >> 10) & 0x1FFFFFu;
  d.f4 = 0;
  return d;
}

__host__ __device__ __forceinline__ Draw site_draw(unsigned long long seed, unsigned long long sweep, uint32_t x,
                                                   uint32_t y, uint32_t z, uint32_t nx, uint32_t ny, bool flip) {
  if (flip) {
    const U4 o = site_draws(seed, sweep, x + nx * (y + ny * z), 0);
    return Draw{o.x >> 8, o.y >> 8, o.z >> 8, o.w >> 8};
  }
  return pair_half(site_draws(seed, sweep, pair_counter(x, y, z, nx, ny), 0), (x >> 1) & 1u);
}

// Field -> uniform in [0, 1): 21-bit fields for pair draws, 24-bit for flip models.
__host__ __device__ __forceinline__ float unif(uint32_t f, bool flip) {
  return (float)f * (flip ? (1.0f / 16777216.0f) : (1.0f / 2097152.0f));
}
__host__ __device__ __forceinline__ double unif_d(uint32_t f, bool flip) {
  return (double)f * (flip ? (1.0 / 16777216.0) : (1.0 / 2097152.0));
}

// Random initial director of one site (stream 2 of the site's Philox counter): successive draws (site, attempt)
// give a point of the grid of odd integers in (-2^24, 2^24)^3; the first one strictly inside the ball of radius
// 2^24 is projected onto the unit sphere. A uniform point of a ball projects to a uniform point of its sphere, and
// the arithmetic is integer products, one IEEE double square root and IEEE double divisions, so host and device
// give the same bits. An attempt is accepted with probability pi / 6; after 64 rejections (probability 1e-21) the
// site takes (0, 0, 1).
__host__ __device__ inline void random_director(unsigned long long seed, uint32_t site, float out[3]) {
  for (uint32_t attempt = 0; attempt < 64; attempt++) {
    const U4 r = site_draws(seed, attempt, site, 2);
    const long long ix = 2ll * (long long)(r.x >> 8) + 1 - 16777216ll;
    const long long iy = 2ll * (long long)(r.y >> 8) + 1 - 16777216ll;
    const long long iz = 2ll * (long long)(r.z >> 8) + 1 - 16777216ll;
    const long long s = ix * ix + iy * iy + iz * iz;  // < 3 * 2^48: exact
    if (s < (1ll << 48)) {
      const double len = sqrt((double)s);  // s < 2^48 is exact in double; sqrt rounds correctly
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

// Rotation axis from the axis field exactly as `u2 < 0.333` / `u2 < 0.666` in double (src/evolve.cpp:156-160):
// for u2 = m 2^-24 the tests are m < 5586813 and m < 11173626, for u2 = m 2^-21 m < 698352 and m < 1396704.
__host__ __device__ __forceinline__ int rotation_axis(uint32_t m, bool flip) {
  const uint32_t t1 = flip ? 5586813u : 698352u, t2 = flip ? 11173626u : 1396704u;
  return m < t1 ? 0 : (m < t2 ? 1 : 2);
}

}  // namespace mcl
