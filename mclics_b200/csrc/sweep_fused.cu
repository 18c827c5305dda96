// Fused two-colour sweep: one pass over HBM per sweep, both colours, measurement fused.
//
// Work item = (replica, x/y tile of TX x TY sites, z segment [z0, z1)). A CTA streams the planes of its segment
// through a ring of NSLOT shared-memory slots, each slot holding one padded plane tile of
// (TX + 8) x (TY + 4) sites x 3 components, loaded by one TMA box copy (4D tensor map over (px, py, nz, 3) of the
// padded SoA buffer; the box starts 4 cells left of the tile so its x coordinate stays 16-byte aligned, and the
// periodic wrap comes from the ghost cells). At step k the CTA
//   (a) updates colour A (x + y + z even) of plane k on the tile plus a one-site ring,
//   (b) updates colour B of plane k - 1 on the tile (all its colour-A neighbours are final after (a)),
//   (c) writes plane k - 1 (both colours final) to the other director buffer, with the ghost copies of edge sites,
//       and adds its site terms to the FP64 observables.
// The ring sites of (a) are recomputed by the neighbouring tiles too; they reproduce the owner's result exactly
// because the trial draws are Philox(seed, sweep, site) and the inputs (old colour-B neighbours) are the same.
// Segment ends load two extra planes on each side (z0 - 2 .. z1 + 1) for the same reason along z.
//
// Energy: every bond has exactly one colour-B end, so E_total = sum_B (2 bond_B + single_B) + sum_A single_A, with
// all terms known when the site is final; Q and sum n are summed at write-out.
//
// Every wait on a TMA barrier is bounded by %globaltimer; on timeout the CTA sets the engine's error word, waits
// (bounded) for its copies in flight and returns, and the host reports MCL_ERR_CUDA.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "fused.h"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {

constexpr int FT = 256;      // threads per CTA
constexpr int NSLOT = 6;     // plane slots (4 live + 2 in flight)
constexpr int kMaxTX = 64, kMaxTY = 32;

struct FusedItem {
  int rep, x0, y0, z0, z1;
};

struct FusedArgs {
  const CUtensorMap *tmaps;     // [n_rep][2] (one per director buffer), 64-byte aligned
  float *out;                   // director buffer written by this sweep
  const RepDesc *reps;
  RepState *st;
  const FusedItem *items;
  double *partials;             // [n_items][kPartials]
  const unsigned long long *sweep_ctr;
  unsigned int *err;            // error word (bit 0: TMA wait timeout)
  int cur;                      // buffer read by this sweep (selects the tensor map)
  int tx, ty;                   // tile size
  long long timeout_ns;
  int skip_first_load;          // test hook: never issue the first TMA load (its wait must time out)
};

struct FusedPlan {
  int tx = 64, ty = 16, seg = 32;
  int n_items = 0;
  FusedItem *d_items = nullptr;
  CUtensorMap *d_tmaps = nullptr;
  double *d_partials = nullptr;
  int *d_first = nullptr;  // first item of each replica (n_rep + 1)
  unsigned int *d_err = nullptr;
  size_t smem = 0;
  long long timeout_ns = 2000000000ll;
  int skip_first_load = 0;
};

// ---- PTX helpers -----------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void tma_load_plane(float *dst, const CUtensorMap *map, int x, int y, int z,
                                               unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait for the barrier's phase `parity`; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((long long)(globaltimer() - t0) > timeout_ns) return false;
  }
}

// ---- the kernel --------------------------------------------------------------------------------------------
// Shared memory: NSLOT plane slots of 3 * (tx + 8) * (ty + 4) floats, then NSLOT mbarriers.
template <int POT, int GEO, bool MEASURE>
__global__ void __launch_bounds__(FT, 2) k_sweep_fused(ModelDev m, FusedArgs a) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = (unsigned char *)(((uintptr_t)smem_dyn + 127) & ~(uintptr_t)127);
  const FusedItem it = a.items[blockIdx.x];
  const RepDesc R = a.reps[it.rep];
  const RepState S = a.st[it.rep];
  const int TX = a.tx, TY = a.ty;
  const int W = TX + 8, H = TY + 4;      // slot row length and rows
  const int plane_floats = W * H;        // one component
  const int slot_floats = ((3 * plane_floats + 31) / 32) * 32;  // slots start on 128-byte boundaries
  float *slots = reinterpret_cast<float *>(smem_raw);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + (size_t)NSLOT * slot_floats * 4);
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  const CUtensorMap *map = a.tmaps + 2 * it.rep + a.cur;
  const unsigned long long sweep = *a.sweep_ctr;
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  const bool perx = R.periodic[0], pery = R.periodic[1], perz = R.periodic[2];
  const int x0 = it.x0, y0 = it.y0, z0 = it.z0, z1 = it.z1;
  const float T = S.T, invT = 1.f / T, av = S.ang_var, elecE = S.elecE;
  const unsigned box_bytes = (unsigned)(3 * plane_floats) * 4u;

  if (tid == 0) {
    s_fail = 0;
    for (int q = 0; q < NSLOT; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
  }
  __syncthreads();

  // plane p (local index lp = p - (z0 - 2)) lives in slot lp % NSLOT; exists unless free z and p outside [0, nz)
  const int pbeg = z0 - 2, pend = z1 + 1;  // inclusive range of planes used
  auto plane_exists = [&](int p) { return perz || (p >= 0 && p < nz); };
  auto wrapz = [&](int p) { return p < 0 ? p + nz : (p >= nz ? p - nz : p); };
  auto issue = [&](int p) {  // called by thread 0 only
    if (p > pend) return;
    const int lp = p - pbeg;
    if (a.skip_first_load && lp == 0) return;  // test hook: nothing will complete this barrier phase
    unsigned long long *bar = &bars[lp % NSLOT];
    if (!plane_exists(p)) {  // no copy: complete the slot's phase anyway, so every slot advances once per use
      mbar_arrive(bar);
      return;
    }
    mbar_expect_tx(bar, box_bytes);
    tma_load_plane(slots + (size_t)(lp % NSLOT) * slot_floats, map, x0, y0, wrapz(p), bar);
  };
  // Slot reuse: at step k the CTA reads planes k-2 .. k+1; plane k+3 goes into the slot of plane k-3, whose last
  // reader was step k-1. Four planes are issued before the loop, one per step after that.
  int last_issued = pbeg - 1;
  if (tid == 0) {
    for (int p = pbeg; p <= pbeg + 3 && p <= pend; p++) issue(p);
    last_issued = min(pend, pbeg + 3);
  }

  auto wait_plane = [&](int p) -> bool {  // every thread waits; returns false if the CTA must bail out
    if (p <= pend && plane_exists(p)) {
      const int lp = p - pbeg;
      const unsigned parity = (unsigned)((lp / NSLOT) & 1);
      if (!mbar_wait_bounded(&bars[lp % NSLOT], parity, a.timeout_ns)) s_fail = 1;
    }
    __syncthreads();
    return s_fail == 0;
  };

  // slot base pointers
  auto slot_of = [&](int p) -> const float * { return slots + (size_t)((p - pbeg) % NSLOT) * slot_floats; };
  auto slot_of_w = [&](int p) -> float * { return slots + (size_t)((p - pbeg) % NSLOT) * slot_floats; };
  // cell (x, y) of the tile's padded window: column x - (x0 - 4), row y - (y0 - 2)
  auto cell = [&](int x, int y) { return (y - y0 + 2) * W + (x - x0 + 4); };

  unsigned accepted = 0;
  double acc_e = 0, acc_q[6] = {0, 0, 0, 0, 0, 0}, acc_n[3] = {0, 0, 0};

  // one trial move of site (x, y, z) (unwrapped coordinates inside the window), director in slot `cur`
  auto update = [&](int x, int y, int z, float *cs, const float *below, const float *above, bool count,
                    float *bond_out, float *single_out) {
    const int c = cell(x, y);
    Vec3 n{cs[c], cs[c + plane_floats], cs[c + 2 * plane_floats]};
    Vec3 nb[6];
    unsigned present = 0;
    const int xw = perx ? (x < 0 ? x + nx : (x >= nx ? x - nx : x)) : x;
    const int yw = pery ? (y < 0 ? y + ny : (y >= ny ? y - ny : y)) : y;
    const int zw = perz ? (z < 0 ? z + nz : (z >= nz ? z - nz : z)) : z;
    // +x, -x, +y, -y in plane; +z (above), -z (below)
    const int offs[4] = {1, -1, W, -W};
#pragma unroll
    for (int d = 0; d < 4; d++) {
      bool ok;
      if (d == 0) ok = perx || xw + 1 < nx;
      else if (d == 1) ok = perx || xw - 1 >= 0;
      else if (d == 2) ok = pery || yw + 1 < ny;
      else ok = pery || yw - 1 >= 0;
      const int q = c + offs[d];
      nb[d] = Vec3{cs[q], cs[q + plane_floats], cs[q + 2 * plane_floats]};
      present |= ok ? (1u << d) : 0u;
    }
    if (above) {
      nb[4] = Vec3{above[c], above[c + plane_floats], above[c + 2 * plane_floats]};
      present |= 16u;
    } else {
      nb[4] = Vec3{0.f, 0.f, 0.f};
    }
    if (below) {
      nb[5] = Vec3{below[c], below[c + plane_floats], below[c + 2 * plane_floats]};
      present |= 32u;
    } else {
      nb[5] = Vec3{0.f, 0.f, 0.f};
    }
    int sid = -1;
    Vec3 s{0.f, 0.f, 0.f};
    if (GEO == GEO_SLAB) {
      float sz;
      sid = slab_surface(zw, nz, sz);
      s.z = sz;
    }
    const uint32_t site = (uint32_t)xw + (uint32_t)nx * ((uint32_t)yw + (uint32_t)ny * (uint32_t)zw);
    const U4 r = site_draws(R.seed, sweep, site, 0);
    const float va = (2.f * u24(r.x) - 1.f) * av;
    const Vec3 nn = rotate_trial(n, va, rotation_axis(r.y));
    const float b_old = bond_sum<POT>(m, n, nb, present), b_new = bond_sum<POT>(m, nn, nb, present);
    float s_old = 0.f, s_new = 0.f;
    if (sid >= 0) {
      s_old = anchoring_energy(m, sid, n, s);
      s_new = anchoring_energy(m, sid, nn, s);
    }
    if (m.field_on) {
      s_old += field_energy(m, n, elecE);
      s_new += field_energy(m, nn, elecE);
    }
    const float e_old = b_old + s_old, e_new = b_new + s_new;
    Vec3 curv = n;
    float e_cur = e_old, b_cur = b_old, s_cur = s_old;
    bool moved = false;
    if (metropolis(u24(r.z), e_new - e_old, invT, T)) {
      curv = nn;
      e_cur = e_new;
      b_cur = b_new;
      s_cur = s_new;
      moved = true;
      if (count) accepted++;
    }
    if (m.flip) {
      const Vec3 f{-curv.x, -curv.y, -curv.z};
      const float bf = bond_sum<POT>(m, f, nb, present);
      float sf = 0.f;
      if (sid >= 0) sf = anchoring_energy(m, sid, f, s);
      if (m.field_on) sf += field_energy(m, f, elecE);
      if (metropolis(u24(r.w), (bf + sf) - e_cur, invT, T)) {
        curv = f;
        b_cur = bf;
        s_cur = sf;
        moved = true;
      }
    }
    if (moved) {
      cs[c] = curv.x;
      cs[c + plane_floats] = curv.y;
      cs[c + 2 * plane_floats] = curv.z;
    }
    if (bond_out) *bond_out = b_cur;
    if (single_out) *single_out = s_cur;
  };

  bool ok = wait_plane(z0 - 2) && wait_plane(z0 - 1);
  // ring limits: sites that exist (free axes) or whose ghost data is valid (periodic axes)
  const int xr_lo = max(x0 - 1, perx ? -1 : 0), xr_hi = min(x0 + TX, perx ? nx : nx - 1);
  const int yr_lo = max(y0 - 1, pery ? -1 : 0), yr_hi = min(y0 + TY, pery ? ny : ny - 1);
  int k = z0 - 1;
  for (; ok && k <= z1; k++) {
    ok = wait_plane(k + 1);  // planes k-2 .. k+1 are resident after this
    if (!ok) break;
    if (tid == 0 && k + 3 <= pend) {
      issue(k + 3);
      last_issued = k + 3;
    }
    // (a) colour A of plane k on the tile plus a one-site ring
    if (plane_exists(k)) {
      float *cs = slot_of_w(k);
      const float *below = plane_exists(k - 1) ? slot_of(k - 1) : nullptr;
      const float *above = plane_exists(k + 1) ? slot_of(k + 1) : nullptr;
      const int rw = TX + 2, nrow = TY + 2, half = (rw + 1) / 2;
      for (int q = tid; q < half * nrow; q += FT) {
        const int row = q / half, j = q % half;
        const int y = y0 - 1 + row;
        const int xs = x0 - 1;
        const int x = xs + 2 * j + ((xs + y + k) & 1);  // parity 0 sites of the row
        if (x < xr_lo || x > xr_hi || y < yr_lo || y > yr_hi) continue;
        const bool interior = x >= x0 && x < x0 + TX && y >= y0 && y < y0 + TY && x < nx && y < ny && k >= z0 &&
                              k < z1;
        update(x, y, k, cs, below, above, interior, nullptr, nullptr);
      }
    }
    __syncthreads();
    // (b) colour B of plane k - 1 (owned planes only), (c) write-out of plane k - 1
    const int pb = k - 1;
    if (pb >= z0 && pb < z1 && plane_exists(pb)) {
      float *cs = slot_of_w(pb);
      const float *below = plane_exists(pb - 1) ? slot_of(pb - 1) : nullptr;
      const float *above = plane_exists(pb + 1) ? slot_of(pb + 1) : nullptr;
      const int half = TX / 2;
      for (int q = tid; q < half * TY; q += FT) {
        const int row = q / half, j = q % half;
        const int y = y0 + row;
        const int x = x0 + 2 * j + ((x0 + y + pb + 1) & 1);  // parity 1 sites
        if (x >= nx || y >= ny) continue;
        float bnd, sgl;
        update(x, y, pb, cs, below, above, true, &bnd, &sgl);
        if (MEASURE) acc_e += (double)(2.f * bnd + sgl);
      }
      __syncthreads();
      // (c) write-out (both colours) and site terms of colour A
      const int zw = pb < 0 ? pb + nz : (pb >= nz ? pb - nz : pb);
      for (int q = tid; q < TX * TY; q += FT) {
        const int row = q / TX, col = q % TX;
        const int y = y0 + row, x = x0 + col;
        if (x >= nx || y >= ny) continue;
        const int c = cell(x, y);
        const float vx = cs[c], vy = cs[c + plane_floats], vz = cs[c + 2 * plane_floats];
        const long long base = R.off + ((long long)zw * R.py) * R.px;
        // the site and its ghost images along periodic axes (x + nx for x < 2, x - nx for x >= nx - 2)
        int xs_[3] = {x, 0, 0}, ys_[3] = {y, 0, 0}, ncx = 1, ncy = 1;
        if (perx) {
          if (x < 2) xs_[ncx++] = x + nx;
          if (x >= nx - 2) xs_[ncx++] = x - nx;
        }
        if (pery) {
          if (y < 2) ys_[ncy++] = y + ny;
          if (y >= ny - 2) ys_[ncy++] = y - ny;
        }
        for (int ix = 0; ix < ncx; ix++)
          for (int iy = 0; iy < ncy; iy++) {
            const long long o = base + (long long)(ys_[iy] + GY) * R.px + (xs_[ix] + GX);
            a.out[o] = vx;
            a.out[o + R.comp] = vy;
            a.out[o + 2 * R.comp] = vz;
          }
        if (MEASURE) {
          const double dx = vx, dy = vy, dz = vz;
          acc_q[0] += 1.5 * dx * dx - 0.5;
          acc_q[1] += 1.5 * dx * dy;
          acc_q[2] += 1.5 * dx * dz;
          acc_q[3] += 1.5 * dy * dy - 0.5;
          acc_q[4] += 1.5 * dy * dz;
          acc_q[5] += 1.5 * dz * dz - 0.5;
          acc_n[0] += dx;
          acc_n[1] += dy;
          acc_n[2] += dz;
          if (((x + y + pb) & 1) == 0) {  // colour A: single-site terms (colour B added 2 bond + single above)
            float sgl = 0.f;
            const Vec3 v{vx, vy, vz};
            if (GEO == GEO_SLAB) {
              float sz;
              const int sid = slab_surface(zw, nz, sz);
              if (sid >= 0) sgl += anchoring_energy(m, sid, v, Vec3{0.f, 0.f, sz});
            }
            if (m.field_on) sgl += field_energy(m, v, elecE);
            acc_e += (double)sgl;
          }
        }
      }
    }
    __syncthreads();  // slot of plane k - 2 is free after this step
  }

  if (!ok) {
    // bail out: record the failure and wait (bounded) for this CTA's loads still in flight
    if (tid == 0) {
      atomicOr(a.err, 1u);
      // loads possibly in flight: the last NSLOT issued planes (one per slot)
      for (int p = max(pbeg, last_issued - NSLOT + 1); p <= last_issued; p++) {
        if (!plane_exists(p) || (a.skip_first_load && p == pbeg)) continue;
        const int lp = p - pbeg;
        mbar_wait_bounded(&bars[lp % NSLOT], (unsigned)((lp / NSLOT) & 1), a.timeout_ns);
      }
    }
    __syncthreads();
    return;
  }

  // reductions: acceptance count and the FP64 partials of this work item
  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&a.st[it.rep].acc, (unsigned long long)wsum);
  if (MEASURE) {
    __shared__ double red[FT / 32][kPartials];
    double v[kPartials] = {acc_e, acc_q[0], acc_q[1], acc_q[2], acc_q[3], acc_q[4], acc_q[5], acc_n[0], acc_n[1], acc_n[2]};
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int k = 0; k < kPartials; k++) {
      double x = v[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) red[warp][k] = x;
    }
    __syncthreads();
    if (tid < kPartials) {
      double x = 0.0;
      for (int w = 0; w < FT / 32; w++) x += red[w][tid];
      a.partials[(long long)blockIdx.x * kPartials + tid] = x;
    }
  }
}

// ---- host side ----------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

bool fused_supported(const mcl_engine *e) {
  if (e->geo != GEO_BULK && e->geo != GEO_SLAB) return false;
  return get_encode() != nullptr;
}

static int encode_map(CUtensorMap *map, float *base, const RepDesc &D, int tx, int ty) {
  cuuint64_t dims[4] = {(cuuint64_t)D.px, (cuuint64_t)D.py, (cuuint64_t)D.nz, 3};
  cuuint64_t strides[3] = {(cuuint64_t)D.px * 4, (cuuint64_t)D.px * D.py * 4, (cuuint64_t)D.comp * 4};
  cuuint32_t box[4] = {(cuuint32_t)(tx + 8), (cuuint32_t)(ty + 4), 1, 3};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = get_encode()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base + D.off, dims, strides, box, es,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MCL_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return MCL_OK;
}

#define CKF(call)                                        \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Tile and segment choice: 64 x 16 tiles (x a multiple of 4 for the TMA box), and z segments sized so that the
// number of work items is close to a multiple of the resident CTAs (2 per SM).
static void choose_tiles(const mcl_engine *e, FusedPlan &P, int sms) {
  P.tx = 64;
  P.ty = 16;
  long long tiles = 0, maxz = 1;
  for (auto &D : e->desc) {
    tiles += (long long)((D.nx + P.tx - 1) / P.tx) * ((D.ny + P.ty - 1) / P.ty);
    maxz = std::max<long long>(maxz, D.nz);
  }
  const long long slots = 2ll * sms;
  // smallest segment count (longest segments) whose item count fills the resident slots about evenly
  int best = 1;
  double best_eff = 0;
  for (int nseg = 1; nseg <= 64; nseg++) {
    long long items = tiles * nseg;
    double waves = (double)items / slots;
    double eff = waves / std::ceil(waves);
    // extra planes per segment cost ~4/seg_len of the reads
    double seg_len = (double)maxz / nseg;
    if (seg_len < 8) break;
    double score = eff * (1.0 - 4.0 / (seg_len + 4.0) * 0.5);
    if (score > best_eff + 1e-9) {
      best_eff = score;
      best = nseg;
    }
  }
  P.seg = (int)((maxz + best - 1) / best);
}

int fused_create(mcl_engine *e) {
  FusedPlan *P = new FusedPlan();
  e->fused = P;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  choose_tiles(e, *P, sms);
  // second director buffer
  CKF(cudaMalloc(&e->d_dir[1], (size_t)e->dir_floats * sizeof(float)));
  CKF(cudaMemsetAsync(e->d_dir[1], 0, (size_t)e->dir_floats * sizeof(float), e->stream));
  // tensor maps
  std::vector<CUtensorMap> maps(2 * e->n_rep);
  for (int r = 0; r < e->n_rep; r++)
    for (int b = 0; b < 2; b++) {
      int rc = encode_map(&maps[2 * r + b], e->d_dir[b], e->desc[r], P->tx, P->ty);
      if (rc) return rc;
    }
  CKF(cudaMalloc(&P->d_tmaps, maps.size() * sizeof(CUtensorMap)));
  CKF(cudaMemcpy(P->d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  // work items, replica-major, then z segment, y tile, x tile
  std::vector<FusedItem> items;
  std::vector<int> first;
  for (int r = 0; r < e->n_rep; r++) {
    first.push_back((int)items.size());
    const RepDesc &D = e->desc[r];
    for (int z0 = 0; z0 < D.nz; z0 += P->seg)
      for (int y0 = 0; y0 < D.ny; y0 += P->ty)
        for (int x0 = 0; x0 < D.nx; x0 += P->tx) items.push_back(FusedItem{r, x0, y0, z0, std::min(D.nz, z0 + P->seg)});
  }
  first.push_back((int)items.size());
  P->n_items = (int)items.size();
  CKF(cudaMalloc(&P->d_items, items.size() * sizeof(FusedItem)));
  CKF(cudaMemcpy(P->d_items, items.data(), items.size() * sizeof(FusedItem), cudaMemcpyHostToDevice));
  CKF(cudaMalloc(&P->d_first, first.size() * sizeof(int)));
  CKF(cudaMemcpy(P->d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice));
  CKF(cudaMalloc(&P->d_partials, (size_t)P->n_items * kPartials * sizeof(double)));
  CKF(cudaMalloc(&P->d_err, sizeof(unsigned int)));
  CKF(cudaMemset(P->d_err, 0, sizeof(unsigned int)));
  const size_t slot_floats = ((size_t)3 * (P->tx + 8) * (P->ty + 4) + 31) / 32 * 32;
  P->smem = 128 + (size_t)NSLOT * slot_floats * sizeof(float) + NSLOT * sizeof(unsigned long long);
  return MCL_OK;
}

void fused_destroy(mcl_engine *e) {
  FusedPlan *P = e->fused;
  if (!P) return;
  cudaFree(P->d_items);
  cudaFree(P->d_tmaps);
  cudaFree(P->d_partials);
  cudaFree(P->d_first);
  cudaFree(P->d_err);
  delete P;
  e->fused = nullptr;
}

template <int POT, int GEO, bool MEAS>
static cudaError_t launch_one(const mcl_engine *e, const FusedArgs &a) {
  auto k = k_sweep_fused<POT, GEO, MEAS>;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->fused->smem);
  if (err != cudaSuccess) return err;
  k<<<e->fused->n_items, FT, e->fused->smem, e->stream>>>(e->model, a);
  return cudaGetLastError();
}

template <int POT, int GEO>
static cudaError_t launch_meas(const mcl_engine *e, const FusedArgs &a, bool measure) {
  return measure ? launch_one<POT, GEO, true>(e, a) : launch_one<POT, GEO, false>(e, a);
}

template <int POT>
static cudaError_t launch_geo(const mcl_engine *e, const FusedArgs &a, bool measure) {
  return e->geo == GEO_SLAB ? launch_meas<POT, GEO_SLAB>(e, a, measure) : launch_meas<POT, GEO_BULK>(e, a, measure);
}

int fused_sweep(mcl_engine *e, bool measure, cudaEvent_t ev0, cudaEvent_t ev1) {
  FusedPlan *P = e->fused;
  FusedArgs a;
  a.tmaps = P->d_tmaps;
  a.out = e->d_dir[e->cur ^ 1];
  a.reps = e->d_desc;
  a.st = e->d_state;
  a.items = P->d_items;
  a.partials = P->d_partials;
  a.sweep_ctr = e->d_sweep;
  a.err = P->d_err;
  a.cur = e->cur;
  a.tx = P->tx;
  a.ty = P->ty;
  a.timeout_ns = P->timeout_ns;
  a.skip_first_load = P->skip_first_load;
  if (ev0) CKF(cudaEventRecord(ev0, e->stream));
  cudaError_t err;
  if (e->model.potential == POT_GHRL)
    err = launch_geo<POT_GHRL>(e, a, measure);
  else if (e->model.potential == POT_PEAR)
    err = launch_geo<POT_PEAR>(e, a, measure);
  else
    err = launch_geo<POT_LL>(e, a, measure);
  if (err != cudaSuccess) return cuda_fail(err, "fused sweep launch");
  if (ev1) CKF(cudaEventRecord(ev1, e->stream));
  e->cur ^= 1;
  e->launches += 2;
  BlockTable t;
  t.first = P->d_first;
  LaunchCtx c = e->ctx();
  CKF(launch_finalize(c, t, P->d_partials, measure ? 1 : 0, e->d_series, e->d_series_len, e->d_done));
  return MCL_OK;
}

int fused_check_error(mcl_engine *e) {
  if (!e->fused) return MCL_OK;
  unsigned int v = 0;
  CKF(cudaMemcpyAsync(&v, e->fused->d_err, sizeof v, cudaMemcpyDeviceToHost, e->stream));
  CKF(cudaStreamSynchronize(e->stream));
  if (v) {
    unsigned int zero = 0;
    CKF(cudaMemcpy(e->fused->d_err, &zero, sizeof zero, cudaMemcpyHostToDevice));
    return fail(MCL_ERR_CUDA, "fused sweep: a TMA load did not complete within %.3f s (error word 0x%x)",
                e->fused->timeout_ns * 1e-9, v);
  }
  return MCL_OK;
}

void fused_set_test_hooks(mcl_engine *e, long long timeout_ns, int skip_first_load) {
  if (!e->fused) return;
  if (timeout_ns > 0) e->fused->timeout_ns = timeout_ns;
  e->fused->skip_first_load = skip_first_load;
}

}  // namespace mcl
