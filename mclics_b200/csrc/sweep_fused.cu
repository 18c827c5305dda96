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

#include <stdlib.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "fused.h"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {

constexpr int FT = 256;      // threads per CTA
constexpr int NSLOT = 6;     // plane slots (4 live + 2 in flight)

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
  int measure;                  // fuse the observables
  long long timeout_ns;
  int skip_first_load;          // test hook: never issue the first TMA load (its wait must time out)
};

// Tile configurations: rows per tile and threads per CTA (64 columns always).
struct FusedCfg {
  int ty, nt, ctas_per_sm;
};
static const FusedCfg kCfgs[] = {{14, 256, 2}, {28, 512, 1}};
constexpr int kNumCfgs = 2;

struct FusedPlan {
  int cfg = 0, tx = 64, ty = 14, seg = 32;
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

__device__ __forceinline__ void tma_load_plane(float *dst, const CUtensorMap *map, int j, int y, int z,
                                               unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(j), "r"(0), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
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
// Tile: TX = 64 columns (32 sites of each x parity) x TY rows. Window in shared memory, per component and row:
// the even-x half-row then the odd-x half-row, 40 cells each (half-row index j0 - 4 .. j0 + 35, j0 = x0 / 2), for
// rows y0 - 2 .. y0 + TY + 1: exactly one 5-D TMA box (40, 2, TY + 4, 1, 3) of the split HBM layout.
constexpr int TXF = 64, HALF = 40, RW = 2 * HALF, NPAIR = 16, NSL = 7;

template <int TY>
struct Win {
  static constexpr int H = TY + 4, PF = RW * H, SLOT = (3 * PF + 31) / 32 * 32;
};

__device__ __forceinline__ float f4get(const float4 &v, int e) {  // e compile-time after unrolling
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// Geometry/boundary facts of a work item that the site updates need.
struct Ctx {
  int nx, ny, nz;
  bool perx, pery;
  unsigned long long seed, sweep;
  float T, invT, av, elecE;
};

// One task: the two sites of half-row h (x parity h) at window half-row cells jb and jb + 1 (jb even), i.e. sites
// x = 2 (j0 - 4 + jb) + h and x + 2 of row y. v0 / v1: whether each is updated. The updated pair goes back to shared
// memory; accepted rotations of counted sites and (2 bond + single) of measured sites are accumulated.
template <int POT, int GEO, bool FLIP, int TY>
__device__ __forceinline__ void pair_task(const ModelDev &m, const Ctx &c, float *cs, const float *below,
                                          const float *above, int wy, int h, int jb, int x, int y, int zw, bool v0,
                                          bool v1, bool count, bool meas, unsigned &accepted, float &e_acc) {
  constexpr int PF = Win<TY>::PF;
  float *own = cs + (wy * 2 + h) * HALF + jb;                 // component 0
  const float *oth = cs + (wy * 2 + (h ^ 1)) * HALF + jb - 1 + h;  // other parity, 3 consecutive cells
  const int up = 2 * HALF, dn = -2 * HALF;                    // same half-row of the next / previous row
  const float *zu = above ? above + (wy * 2 + h) * HALF + jb : own;
  const float *zd = below ? below + (wy * 2 + h) * HALF + jb : own;
  float2 o[3], yu[3], yd[3], pu[3], pd[3];
  float xa[3], xb[3], xc[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    o[q] = *reinterpret_cast<const float2 *>(own + q * PF);
    yu[q] = *reinterpret_cast<const float2 *>(own + q * PF + up);
    yd[q] = *reinterpret_cast<const float2 *>(own + q * PF + dn);
    pu[q] = *reinterpret_cast<const float2 *>(zu + q * PF);
    pd[q] = *reinterpret_cast<const float2 *>(zd + q * PF);
    xa[q] = oth[q * PF];
    xb[q] = oth[q * PF + 1];
    xc[q] = oth[q * PF + 2];
  }
  int sid = -1;
  Vec3 sn{0.f, 0.f, 0.f};
  if (GEO == GEO_SLAB) {
    float sz;
    sid = slab_surface(zw, c.nz, sz);
    sn.z = sz;
  }
  const int yw = c.pery ? (y < 0 ? y + c.ny : (y >= c.ny ? y - c.ny : y)) : y;
  const float wyp = (c.pery || y + 1 < c.ny) ? 1.f : 0.f, wym = (c.pery || y - 1 >= 0) ? 1.f : 0.f;
  const float wzu = above ? 1.f : 0.f, wzd = below ? 1.f : 0.f;
  const int xs1 = x + 2;
  int xw0 = x, xw1 = xs1;
  if (c.perx) {
    xw0 = x < 0 ? x + c.nx : (x >= c.nx ? x - c.nx : x);
    xw1 = xs1 < 0 ? xs1 + c.nx : (xs1 >= c.nx ? xs1 - c.nx : xs1);
  }
  Draw d0, d1;
  if (FLIP) {
    d0 = site_draw(c.seed, c.sweep, xw0, yw, zw, c.nx, c.ny, true);
    d1 = site_draw(c.seed, c.sweep, xw1, yw, zw, c.nx, c.ny, true);
  } else {
    // one Philox call serves both sites (x & ~2 is shared) unless a periodic wrap split a ring pair
    const U4 out = site_draws(c.seed, c.sweep, pair_counter(v0 ? xw0 : xw1, yw, zw, c.nx, c.ny), 0);
    d0 = pair_half(out, (xw0 >> 1) & 1u);
    d1 = pair_half(out, (xw1 >> 1) & 1u);
  }
  const LaneDraw<float2> ld = lane_draw(d0, d1, FLIP);
  // lane 0: site x, lane 1: site x + 2
  const V3<float2> n{o[0], o[1], o[2]};
  const V3<float2> nb[6] = {
      V3<float2>{make_float2(xb[0], xc[0]), make_float2(xb[1], xc[1]), make_float2(xb[2], xc[2])},  // +x
      V3<float2>{make_float2(xa[0], xb[0]), make_float2(xa[1], xb[1]), make_float2(xa[2], xb[2])},  // -x
      V3<float2>{yu[0], yu[1], yu[2]},
      V3<float2>{yd[0], yd[1], yd[2]},
      V3<float2>{pu[0], pu[1], pu[2]},
      V3<float2>{pd[0], pd[1], pd[2]}};
  float2 wxp = make_float2(1.f, 1.f), wxm = make_float2(1.f, 1.f);
  if (!c.perx) {
    wxp = make_float2(x + 1 < c.nx ? 1.f : 0.f, xs1 + 1 < c.nx ? 1.f : 0.f);
    wxm = make_float2(x - 1 >= 0 ? 1.f : 0.f, xs1 - 1 >= 0 ? 1.f : 0.f);
  }
  const float2 w[6] = {wxp, wxm, make_float2(wyp, wyp), make_float2(wym, wym), make_float2(wzu, wzu),
                       make_float2(wzd, wzd)};
  const SiteResultT<float2> r = site_update<POT, FLIP, float2>(m, n, nb, w, sid, sn, c.elecE, ld, c.av, c.T, c.invT);
  if (v0 | v1) {
    const float2 nx2[3] = {r.n.x, r.n.y, r.n.z};
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const float2 v = make_float2(v0 ? nx2[q].x : o[q].x, v1 ? nx2[q].y : o[q].y);
      *reinterpret_cast<float2 *>(own + q * PF) = v;
    }
  }
  if (count) accepted += (v0 && r.rot.x ? 1u : 0u) + (v1 && r.rot.y ? 1u : 0u);
  if (meas) {
    const float2 eb = __ffma2_rn(make_float2(2.f, 2.f), r.bond, r.single);
    if (v0) e_acc += eb.x;
    if (v1) e_acc += eb.y;
  }
}

template <int POT, int GEO, bool FLIP, int TY, int NT>
__global__ void __launch_bounds__(NT, NT <= 256 ? 2 : 1) k_sweep_fused(ModelDev m, FusedArgs a) {
  constexpr int PF = Win<TY>::PF, SLOT = Win<TY>::SLOT, H = Win<TY>::H;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = (unsigned char *)(((uintptr_t)smem_dyn + 127) & ~(uintptr_t)127);
  float *slots = reinterpret_cast<float *>(smem_raw);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + (size_t)NSL * SLOT * 4);
  __shared__ int s_fail;
  const FusedItem it = a.items[blockIdx.x];
  const RepDesc R = a.reps[it.rep];
  const RepState S = a.st[it.rep];
  const int tid = threadIdx.x;
  const CUtensorMap *map = a.tmaps + 2 * it.rep + a.cur;
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  const bool perz = R.periodic[2];
  const int x0 = it.x0, y0 = it.y0, z0 = it.z0, z1 = it.z1;
  const int j0 = x0 >> 1;
  const bool measure = a.measure != 0;
  Ctx c;
  c.nx = nx;
  c.ny = ny;
  c.nz = nz;
  c.perx = R.periodic[0];
  c.pery = R.periodic[1];
  c.seed = R.seed;
  c.sweep = *a.sweep_ctr;
  c.T = S.T;
  c.invT = 1.f / S.T;
  c.av = S.ang_var;
  c.elecE = S.elecE;
  constexpr unsigned box_bytes = 3u * PF * 4u;

  if (tid == 0) {
    s_fail = 0;
    for (int q = 0; q < NSL; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
  }
  __syncthreads();

  // Plane p (local index lp = p - pbeg) lives in slot lp % NSL; every use of a slot completes one barrier phase.
  const int pbeg = z0 - 2, pend = z1 + 1;
  auto plane_exists = [&](int p) { return perz || (p >= 0 && p < nz); };
  auto wrapz = [&](int p) { return p < 0 ? p + nz : (p >= nz ? p - nz : p); };
  auto slot_ptr = [&](int p) -> float * { return slots + (size_t)((p - pbeg) % NSL) * SLOT; };
  int last_issued = pbeg - 1;  // meaningful in thread 0 only
  auto issue = [&](int p) {    // thread 0 only
    if (p > pend) return;
    const int lp = p - pbeg;
    last_issued = p;
    if (a.skip_first_load && lp == 0) return;  // test hook: nothing will complete this barrier phase
    unsigned long long *bar = &bars[lp % NSL];
    if (!plane_exists(p)) {  // no copy: complete the slot's phase anyway
      mbar_arrive(bar);
      return;
    }
    mbar_expect_tx(bar, box_bytes);
    tma_load_plane(slot_ptr(p), map, j0, y0, wrapz(p), bar);
  };
  int waited = pbeg - 1;  // uniform: highest plane waited for successfully
  auto wait_plane = [&](int p) -> bool {
    if (p <= pend && p > waited) {
      const int lp = p - pbeg;
      if (plane_exists(p) && !mbar_wait_bounded(&bars[lp % NSL], (unsigned)((lp / NSL) & 1), a.timeout_ns)) s_fail = 1;
    }
    __syncthreads();
    if (s_fail) return false;
    if (p > waited) waited = p;
    return true;
  };
  // Slot reuse: at step k the CTA reads planes k-3 .. k+1; plane k+3 goes into the slot of plane k-4, whose last
  // reader was step k-1 (the barrier at the start of step k separates them).
  if (tid == 0)
    for (int p = pbeg; p <= pbeg + 3; p++) issue(p);

  unsigned accepted = 0;
  double dacc[kPartials];
#pragma unroll
  for (int q = 0; q < kPartials; q++) dacc[q] = 0.0;

  // ring columns (colour A of owned planes): left x0 - 1, right min(x0 + TX, nx) (periodic) / x0 + TX (free)
  const bool has_left = c.perx || x0 >= 1;
  const int xright = c.perx ? min(x0 + TXF, nx) : x0 + TXF;
  const bool has_right = xright < nx || (c.perx && xright == nx);
  const int ylo_ring = c.pery ? -1 : 0, yhi_ring = c.pery ? ny : ny - 1;

  bool ok = wait_plane(z0 - 2) && wait_plane(z0 - 1);
  for (int k = z0 - 1; ok && k <= z1 + 2; k++) {
    ok = wait_plane(k + 1);
    if (!ok) break;
    if (tid == 0) issue(k + 3);
    // ---- phase: colour A of plane k, colour B of plane k - 2 (independent), then write-out of plane k - 3
    const bool doA = k <= z1 && plane_exists(k);
    const bool ownA = k >= z0 && k < z1;
    const int kb = k - 2;
    const bool doB = kb >= z0 && kb < z1 && plane_exists(kb);
    const int rowsA = doA ? (ownA ? TY + 2 : TY) : 0;
    const int row0A = ownA ? y0 - 1 : y0;
    const int nAg = rowsA * NPAIR;
    const int nAc = (doA && ownA) ? TY : 0;  // TY/2 ring sites on each side
    const int nB = doB ? TY * NPAIR : 0;
    const int ntask = nAg + nAc + nB;
    const int zwA = wrapz(k), zwB = wrapz(kb);
    float *csA = doA ? slot_ptr(k) : nullptr;
    const float *belowA = (doA && plane_exists(k - 1)) ? slot_ptr(k - 1) : nullptr;
    const float *aboveA = (doA && plane_exists(k + 1)) ? slot_ptr(k + 1) : nullptr;
    float *csB = doB ? slot_ptr(kb) : nullptr;
    const float *belowB = (doB && plane_exists(kb - 1)) ? slot_ptr(kb - 1) : nullptr;
    const float *aboveB = (doB && plane_exists(kb + 1)) ? slot_ptr(kb + 1) : nullptr;
    float eB = 0.f;
    for (int t = tid; t < ntask; t += NT) {
      float *cs;
      const float *below, *above;
      int y, x, h, jb, zw;
      bool v0, v1, count, meas;
      if (t < nAg) {
        const int rr = t / NPAIR, p = t % NPAIR;
        y = row0A + rr;
        h = (y + k) & 1;  // colour A: x + y + k even
        jb = 4 + 2 * p;
        x = x0 + 4 * p + h;
        const bool yok = ownA ? (y >= ylo_ring && y <= yhi_ring) : (y < ny);
        v0 = yok && x < nx;
        v1 = yok && x + 2 < nx;
        cs = csA;
        below = belowA;
        above = aboveA;
        zw = zwA;
        count = ownA && y >= y0 && y < y0 + TY && y < ny;
        meas = false;
      } else if (t < nAg + nAc) {
        // ring columns, one site each (left side first)
        const int q = t - nAg, side = q / (TY / 2), jr = q % (TY / 2);
        const int xcol = side == 0 ? x0 - 1 : xright;
        y = y0 + 2 * jr + ((xcol + y0 + k) & 1);  // (xcol + y + k) even
        const bool valid = (side == 0 ? has_left : has_right) && y < y0 + TY && y < ny;
        h = xcol & 1;
        const int jj = (xcol >> 1) - j0 + 4;  // window cell of the site
        jb = jj & ~1;
        x = xcol - 2 * (jj & 1);  // x of the pair's first site
        v0 = valid && (jj & 1) == 0;
        v1 = valid && (jj & 1) == 1;
        cs = csA;
        below = belowA;
        above = aboveA;
        zw = zwA;
        count = false;
        meas = false;
      } else {
        const int tb = t - nAg - nAc;
        const int rr = tb / NPAIR, p = tb % NPAIR;
        y = y0 + rr;
        h = (y + kb + 1) & 1;  // colour B: x + y + kb odd
        jb = 4 + 2 * p;
        x = x0 + 4 * p + h;
        v0 = y < ny && x < nx;
        v1 = y < ny && x + 2 < nx;
        cs = csB;
        below = belowB;
        above = aboveB;
        zw = zwB;
        count = true;
        meas = measure;
      }
      pair_task<POT, GEO, FLIP, TY>(m, c, cs, below, above, y - y0 + 2, h, jb, x, y, zw, v0, v1, count, meas, accepted,
                                    eB);
    }
    if (measure) dacc[0] += (double)eB;
    // ---- write-out of plane k - 3 (both colours final): rows x halves x 8 chunks of 4 cells
    const int kw = k - 3;
    if (kw >= z0 && kw < z1 && plane_exists(kw)) {
      const float *cw = slot_ptr(kw);
      const int zw = wrapz(kw);
      const long long pbase = R.off + (long long)zw * R.py * R.px;
      int sid = -1;
      float sz = 0.f;
      if (GEO == GEO_SLAB) sid = slab_surface(zw, nz, sz);
      for (int t = tid; t < TY * 16; t += NT) {
        const int rr = t >> 4, h = (t >> 3) & 1, q4 = t & 7;
        const int y = y0 + rr;
        const int jl = j0 + 4 * q4;  // first half-row index of the chunk
        const int xfirst = 2 * jl + h;
        if (y >= ny || xfirst >= nx) continue;
        const int cell = ((rr + 2) * 2 + h) * HALF + 4 + 4 * q4;
        float4 v[3];
#pragma unroll
        for (int q = 0; q < 3; q++) v[q] = *reinterpret_cast<const float4 *>(cw + q * PF + cell);
        const bool full = xfirst + 6 < nx;
        // the row itself, then its ghost copies along a periodic y (y + ny for y < 2, y - ny for y >= ny - 2)
        const bool g1 = c.pery && y < 2, g2 = c.pery && y >= ny - 2;
#pragma unroll
        for (int iy = 0; iy < 3; iy++) {
          if ((iy == 1 && !g1) || (iy == 2 && !g2)) continue;
          const int yy = iy == 0 ? y : (iy == 1 ? y + ny : y - ny);
          float *rowp = a.out + pbase + (long long)(yy + GY) * R.px + h * R.hp + GH;  // half-row, j = 0
          float *dst = rowp + jl;
          if (full) {
#pragma unroll
            for (int q = 0; q < 3; q++) *reinterpret_cast<float4 *>(dst + q * R.comp) = v[q];
          } else {
#pragma unroll
            for (int e = 0; e < 4; e++)
              if (xfirst + 2 * e < nx)
#pragma unroll
                for (int q = 0; q < 3; q++) dst[q * R.comp + e] = f4get(v[q], e);
          }
          if (c.perx) {  // ghost columns: x + nx for x < 2 (half index nx/2), x - nx for x >= nx - 2 (index -1)
            if (jl == 0)
#pragma unroll
              for (int q = 0; q < 3; q++) rowp[q * R.comp + (nx >> 1)] = v[q].x;
            const int el = (nx >> 1) - 1 - jl;  // element holding half index nx/2 - 1 (nx is even when periodic)
            if (el >= 0 && el < 4)
#pragma unroll
              for (int q = 0; q < 3; q++) rowp[q * R.comp - 1] = el == 0 ? v[q].x : (el == 1 ? v[q].y : (el == 2 ? v[q].z : v[q].w));
          }
        }
        if (measure) {
          float f[kPartials];
#pragma unroll
          for (int q = 0; q < kPartials; q++) f[q] = 0.f;
          const bool colourA = ((h + y + kw) & 1) == 0;
          const bool single = colourA && (sid >= 0 || m.field_on);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            if (xfirst + 2 * e >= nx) continue;
            const float vx = f4get(v[0], e), vy = f4get(v[1], e), vz = f4get(v[2], e);
            f[1] = fmaf(1.5f * vx, vx, f[1] - 0.5f);
            f[2] = fmaf(1.5f * vx, vy, f[2]);
            f[3] = fmaf(1.5f * vx, vz, f[3]);
            f[4] = fmaf(1.5f * vy, vy, f[4] - 0.5f);
            f[5] = fmaf(1.5f * vy, vz, f[5]);
            f[6] = fmaf(1.5f * vz, vz, f[6] - 0.5f);
            f[7] += vx;
            f[8] += vy;
            f[9] += vz;
            if (single) f[0] += single_energy(m, Vec3{vx, vy, vz}, sid, Vec3{0.f, 0.f, sz}, c.elecE);
          }
#pragma unroll
          for (int q = 0; q < kPartials; q++) dacc[q] += (double)f[q];
        }
      }
    }
  }

  if (!ok) {
    if (tid == 0) {
      atomicOr(a.err, 1u);
      for (int p = max(waited + 1, last_issued - NSL + 1); p <= last_issued; p++) {
        if (!plane_exists(p) || (a.skip_first_load && p == pbeg)) continue;
        const int lp = p - pbeg;
        mbar_wait_bounded(&bars[lp % NSL], (unsigned)((lp / NSL) & 1), a.timeout_ns);
      }
    }
    __syncthreads();
    return;
  }
  (void)H;

  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&a.st[it.rep].acc, (unsigned long long)wsum);
  if (measure) {
    __shared__ double red[NT / 32][kPartials];
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < kPartials; q++) {
      double x = dacc[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) red[warp][q] = x;
    }
    __syncthreads();
    if (tid < kPartials) {
      double x = 0.0;
      for (int w = 0; w < NT / 32; w++) x += red[w][tid];
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

static int encode_map(CUtensorMap *map, float *base, const RepDesc &D, int ty) {
  // 5-D view of the split layout: (half-row cell, x parity, padded row, plane, component)
  cuuint64_t dims[5] = {(cuuint64_t)D.hp, 2, (cuuint64_t)D.py, (cuuint64_t)D.nz, 3};
  cuuint64_t strides[4] = {(cuuint64_t)D.hp * 4, (cuuint64_t)D.px * 4, (cuuint64_t)D.px * D.py * 4, (cuuint64_t)D.comp * 4};
  cuuint32_t box[5] = {(cuuint32_t)HALF, 2, (cuuint32_t)(ty + 4), 1, 3};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = get_encode()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base + D.off, dims, strides, box, es,
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

// Tile and segment choice for configuration `cfg`: z segments sized so that the number of work items is close to
// a multiple of the resident CTAs, with segments long enough that the four extra planes of each stay cheap.
static void choose_segments(const mcl_engine *e, FusedPlan &P, int sms) {
  const FusedCfg &C = kCfgs[P.cfg];
  P.tx = TXF;
  P.ty = C.ty;
  long long tiles = 0, maxz = 1;
  for (auto &D : e->desc) {
    tiles += (long long)((D.nx + P.tx - 1) / P.tx) * ((D.ny + P.ty - 1) / P.ty);
    maxz = std::max<long long>(maxz, D.nz);
  }
  const long long slots = (long long)C.ctas_per_sm * sms;
  int best = 1;
  double best_score = -1;
  for (int nseg = 1; nseg <= 256; nseg++) {
    const double seg_len = (double)maxz / nseg;
    if (seg_len < 6 && nseg > 1) break;
    const long long items = tiles * nseg;
    const double waves = (double)items / slots;
    const double eff = waves / std::ceil(waves);
    const double score = eff * seg_len / (seg_len + 4.0 * 0.35);  // extra planes mostly hit L2
    if (score > best_score + 1e-9) {
      best_score = score;
      best = nseg;
    }
  }
  P.seg = (int)((maxz + best - 1) / best);
}

static int choose_cfg(const mcl_engine *e) {
  // smaller lattices (few tiles) favour the 2-CTA configuration; large planes the 30-row tiles
  long long area = 0;
  for (auto &D : e->desc) area += (long long)D.nx * D.ny;
  const char *env = getenv("MCL_FUSED_CFG");
  if (env) return std::max(0, std::min(kNumCfgs - 1, atoi(env)));
  return area >= 128ll * 128 ? 1 : 0;
}

static int build_items(mcl_engine *e, FusedPlan *P) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  choose_segments(e, *P, sms);
  std::vector<CUtensorMap> maps(2 * e->n_rep);
  for (int r = 0; r < e->n_rep; r++)
    for (int b = 0; b < 2; b++) {
      int rc = encode_map(&maps[2 * r + b], e->d_dir[b], e->desc[r], P->ty);
      if (rc) return rc;
    }
  cudaFree(P->d_tmaps);
  cudaFree(P->d_items);
  cudaFree(P->d_first);
  cudaFree(P->d_partials);
  CKF(cudaMalloc(&P->d_tmaps, maps.size() * sizeof(CUtensorMap)));
  CKF(cudaMemcpy(P->d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
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
  const size_t slot_floats = ((size_t)3 * RW * (P->ty + 4) + 31) / 32 * 32;
  P->smem = 128 + (size_t)NSL * slot_floats * sizeof(float) + NSL * sizeof(unsigned long long);
  return MCL_OK;
}

int fused_create(mcl_engine *e) {
  FusedPlan *P = new FusedPlan();
  e->fused = P;
  P->cfg = choose_cfg(e);
  CKF(cudaMalloc(&e->d_dir[1], (size_t)e->dir_floats * sizeof(float)));
  CKF(cudaMemsetAsync(e->d_dir[1], 0, (size_t)e->dir_floats * sizeof(float), e->stream));
  CKF(cudaMalloc(&P->d_err, sizeof(unsigned int)));
  CKF(cudaMemset(P->d_err, 0, sizeof(unsigned int)));
  return build_items(e, P);
}

int fused_set_cfg(mcl_engine *e, int cfg) {
  if (!e->fused) return fail(MCL_ERR_STATE, "this engine does not use the fused tiled sweep");
  if (cfg < 0 || cfg >= kNumCfgs) return fail(MCL_ERR_ARG, "tile configuration %d outside 0..%d", cfg, kNumCfgs - 1);
  CKF(cudaStreamSynchronize(e->stream));
  e->fused->cfg = cfg;
  return build_items(e, e->fused);
}

int fused_get_cfg(const mcl_engine *e, int *cfg, int *ty, int *seg, int *items) {
  if (!e->fused) return fail(MCL_ERR_STATE, "this engine does not use the fused tiled sweep");
  if (cfg) *cfg = e->fused->cfg;
  if (ty) *ty = e->fused->ty;
  if (seg) *seg = e->fused->seg;
  if (items) *items = e->fused->n_items;
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

template <int POT, int GEO, bool FLIP, int TY, int NT>
static cudaError_t launch_one(const mcl_engine *e, const FusedArgs &a) {
  auto k = k_sweep_fused<POT, GEO, FLIP, TY, NT>;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->fused->smem);
  if (err != cudaSuccess) return err;
  k<<<e->fused->n_items, NT, e->fused->smem, e->stream>>>(e->model, a);
  return cudaGetLastError();
}

template <int POT, int GEO, bool FLIP>
static cudaError_t launch_cfg(const mcl_engine *e, const FusedArgs &a) {
  switch (e->fused->cfg) {
    case 1: return launch_one<POT, GEO, FLIP, 28, 512>(e, a);
    default: return launch_one<POT, GEO, FLIP, 14, 256>(e, a);
  }
}

template <int POT, int GEO>
static cudaError_t launch_flip(const mcl_engine *e, const FusedArgs &a) {
  if (POT == POT_PEAR) return launch_cfg<POT, GEO, true>(e, a);
  return e->model.flip ? launch_cfg<POT, GEO, true>(e, a) : launch_cfg<POT, GEO, false>(e, a);
}

template <int POT>
static cudaError_t launch_geo(const mcl_engine *e, const FusedArgs &a) {
  return e->geo == GEO_SLAB ? launch_flip<POT, GEO_SLAB>(e, a) : launch_flip<POT, GEO_BULK>(e, a);
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
  a.measure = measure ? 1 : 0;
  a.timeout_ns = P->timeout_ns;
  a.skip_first_load = P->skip_first_load;
  if (ev0) CKF(cudaEventRecord(ev0, e->stream));
  cudaError_t err;
  if (e->model.potential == POT_GHRL)
    err = launch_geo<POT_GHRL>(e, a);
  else if (e->model.potential == POT_PEAR)
    err = launch_geo<POT_PEAR>(e, a);
  else
    err = launch_geo<POT_LL>(e, a);
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
