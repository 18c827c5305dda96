// Fused two-colour sweep: one pass over HBM per sweep, both colours, measurement fused.
//
// Work item = (replica, x/y tile of 64 x TY sites, z segment [z0, z1)). A CTA streams the planes of its segment
// through a ring of NSL shared-memory slots. Each slot holds one plane window: per component and row, the even-x
// half-row then the odd-x half-row (40 cells each, half-row index j0 - 4 .. j0 + 35, j0 = x0 / 2), rows y0 - 2 ..
// y0 + TY + 1 — exactly one 5-D TMA box (40, 2, TY + 4, 1, 3) of the split HBM layout (common.cuh), whose x start
// is 16-byte aligned and whose periodic wrap comes from the ghost cells. At plane step k the CTA does, in one phase
// without a barrier between them (the three touch disjoint data):
//   A: colour A (x + y + k even) of plane k on the tile plus the one-site ring its colour-B sites need,
//   B: colour B of plane k - 2 on the tile (its colour-A neighbours in planes k-3 .. k-1 are final),
//   W: write-out of plane k - 3 (both colours final) to the other director buffer, with the ghost copies of edge
//      sites, and its site terms for the FP64 observables.
// Ring sites are recomputed identically by the neighbouring tiles (trial draws are Philox(seed, sweep, site) and the
// inputs, old colour-B neighbours, are the same), so CTAs never communicate. Segment ends load two extra planes on
// each side (z0 - 2 .. z1 + 1) for the same reason along z.
//
// Every task updates the two sites of one colour at x and x + 2 of a row: adjacent cells of one half-row, loaded with
// 8-byte shared loads, computed as float2 lanes with paired FP32 instructions, and sharing one Philox call.
//
// Energy without a second pass: every bond has exactly one colour-B end, so
// E_total = sum_B (2 bond_B + single_B) + sum_A single_A, with all terms known when the site is final.
//
// Every wait on a TMA barrier is bounded by %globaltimer; on timeout the CTA sets the error word, waits (bounded)
// for its copies in flight and returns, and the host reports MCL_ERR_CUDA.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {

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
  int colour;                   // colour-pass kernel: the colour updated (0: x + y + z even)
};

constexpr int TXF = 64, HALF = 40, RW = 2 * HALF, NPAIR = 16, NSL = 7;

template <int TY>
struct Win {
  static constexpr int H = TY + 4, PF = RW * H, SLOT = (3 * PF + 31) / 32 * 32;
};

// ---- PTX helpers -----------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// The dynamic shared-memory window rounded up to 128 bytes, as an offset from the shared array itself: the
// compiler keeps the shared address space (LDS/STS; an integer round trip would make every access generic).
__device__ __forceinline__ unsigned char *smem_align128(unsigned char *base) {
  return base + ((128u - (smem_u32(base) & 127u)) & 127u);
}

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

// One plane window of the split layout: 5-D box at (half-row cell j, parity 0, padded row y, plane z, component 0).
__device__ __forceinline__ void tma_load_plane(float *dst, const CUtensorMap *map, int j, int y, int z,
                                               unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(j), "r"(0), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
      : "memory");
}

// try_wait with a suspend-time hint: a thread whose phase is not complete sleeps (up to hint_ns) instead of
// returning at once, so waiting warps take no issue slots.
__device__ __forceinline__ bool mbar_try_wait_sleep(unsigned long long *bar, unsigned parity, unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Bounded wait for the barrier's phase `parity`; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (true) {
    if (mbar_try_wait_sleep(bar, parity, 100000u)) return true;
    if ((long long)(globaltimer() - t0) > timeout_ns) return false;
  }
}

__device__ __forceinline__ float f4get(const float4 &v, int e) {  // e is compile-time after unrolling
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// Facts of a work item that the site updates need.
struct Ctx {
  int nx, ny, nz;
  bool perx, pery;
  unsigned long long seed, sweep;
  float T, invT, av, elecE;
};

// One task: the two sites of x parity h in window cells jb, jb + 1 (jb even) of window row wy — sites x and x + 2
// of row y. v0 / v1: whether each is updated. The pair goes back to shared memory; accepted rotations of counted
// sites and (2 bond + single) of measured sites are accumulated.
template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY>
__device__ __forceinline__ void pair_task(const ModelDev &m, const Ctx &c, float *cs, const float *below,
                                          const float *above, int wy, int h, int jb, int x, int y, int zw, bool v0,
                                          bool v1, bool count, bool meas, unsigned &accepted, float &e_acc) {
  constexpr int PF = Win<TY>::PF;
  float *own = cs + (wy * 2 + h) * HALF + jb;                      // component 0
  const float *oth = cs + (wy * 2 + (h ^ 1)) * HALF + jb - 1 + h;  // other parity: 3 consecutive cells
  const float *zu = above ? above + (wy * 2 + h) * HALF + jb : own;
  const float *zd = below ? below + (wy * 2 + h) * HALF + jb : own;
  float2 o[3], yu[3], yd[3], pu[3], pd[3];
  float xa[3], xb[3], xc[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    o[q] = *reinterpret_cast<const float2 *>(own + q * PF);
    yu[q] = *reinterpret_cast<const float2 *>(own + q * PF + RW);
    yd[q] = *reinterpret_cast<const float2 *>(own + q * PF - RW);
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
  const int xs1 = x + 2;
  int xw0 = x, xw1 = xs1;
  if (PXY || c.perx) {
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
  float2 w[6];
  if (PXY) {
    w[0] = w[1] = w[2] = w[3] = make_float2(1.f, 1.f);
  } else {
    const float wyp = (c.pery || y + 1 < c.ny) ? 1.f : 0.f, wym = (c.pery || y - 1 >= 0) ? 1.f : 0.f;
    w[0] = make_float2((c.perx || x + 1 < c.nx) ? 1.f : 0.f, (c.perx || xs1 + 1 < c.nx) ? 1.f : 0.f);
    w[1] = make_float2((c.perx || x - 1 >= 0) ? 1.f : 0.f, (c.perx || xs1 - 1 >= 0) ? 1.f : 0.f);
    w[2] = make_float2(wyp, wyp);
    w[3] = make_float2(wym, wym);
  }
  const float wzu = above ? 1.f : 0.f, wzd = below ? 1.f : 0.f;
  w[4] = make_float2(wzu, wzu);
  w[5] = make_float2(wzd, wzd);
  const SiteResultT<float2> r =
      site_update<POT, FLIP, PXY, CHIRAL, FIELD, float2>(m, n, nb, w, sid, sn, c.elecE, ld, c.av, c.T, c.invT);
  const float2 nx2[3] = {r.n.x, r.n.y, r.n.z};
  // Only the updated lanes go back: along a periodic x with nx % 4 == 2 the right ring site shares its pair of cells
  // with the tile's last row pair, whose second lane is outside the lattice — two tasks, one lane each.
  if (v0 && v1) {
#pragma unroll
    for (int q = 0; q < 3; q++) *reinterpret_cast<float2 *>(own + q * PF) = nx2[q];
  } else {
#pragma unroll
    for (int q = 0; q < 3; q++) own[q * PF + (v0 ? 0 : 1)] = v0 ? nx2[q].x : nx2[q].y;
  }
  if (count) accepted += (v0 && r.rot.x ? 1u : 0u) + (v1 && r.rot.y ? 1u : 0u);
  if (meas) {
    const float2 eb = __ffma2_rn(make_float2(2.f, 2.f), r.bond, r.single);
    if (v0) e_acc += eb.x;
    if (v1) e_acc += eb.y;
  }
}

// Static task slots: a thread owns task indices tid and tid + NT of the list [ A rows y0-1 .. y0+TY (16 pairs each)
// | A ring columns (TY sites) | B rows y0 .. y0+TY-1 (16 pairs each) ].
struct TaskSlot {
  int type;  // 0 A row pair, 1 A ring site, 2 B row pair, -1 none
  int rr;    // row offset (A: y = y0 - 1 + rr; B: y = y0 + rr; ring: pair index along the column)
  int p;     // pair index in the row (A, B) or side (ring: 0 left, 1 right)
};

template <int TY>
__device__ __forceinline__ TaskSlot make_slot(int q) {
  constexpr int NAG = (TY + 2) * NPAIR, NAC = TY, NB = TY * NPAIR;
  TaskSlot s;
  if (q < NAG) {
    s.type = 0;
    s.rr = q / NPAIR;
    s.p = q % NPAIR;
  } else if (q < NAG + NAC) {
    s.type = 1;
    s.p = (q - NAG) / (TY / 2);
    s.rr = (q - NAG) % (TY / 2);
  } else if (q < NAG + NAC + NB) {
    s.type = 2;
    s.rr = (q - NAG - NAC) / NPAIR;
    s.p = (q - NAG - NAC) % NPAIR;
  } else {
    s.type = -1;
    s.rr = s.p = 0;
  }
  return s;
}

// Four cells of one half-row chunk, all three components (16-byte stores when the chunk is inside the lattice;
// `room` = nx - x of the chunk's first site, so element e exists when 2 e < room).
__device__ __forceinline__ void write_chunk(float *dst, long long cs, const float4 (&v)[3], bool full, int room) {
  if (full) {
#pragma unroll
    for (int q = 0; q < 3; q++) *reinterpret_cast<float4 *>(dst + q * cs) = v[q];
  } else {
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (2 * e < room)
#pragma unroll
        for (int q = 0; q < 3; q++) dst[q * cs + e] = f4get(v[q], e);
  }
}

// Ghost copies of an edge chunk: along a periodic y the whole chunk again at rows y + ny (y < 2) and y - ny
// (y >= ny - 2); along a periodic x, on each of those rows, x + nx for x < 2 (half index nx / 2) and x - nx for
// x >= nx - 2 (half index -1). row0: the chunk's own half-row at half index 0.
static __device__ __noinline__ void write_ghosts(float *row0, long long cs, int px, float4 v0, float4 v1, float4 v2,
                                                 bool full, int room, int jl, int nx, int ny, int y, bool perx,
                                                 bool pery) {
  const float4 v[3] = {v0, v1, v2};
  for (int iy = 0; iy < 3; iy++) {
    if (iy == 1 && !(pery && y < 2)) continue;
    if (iy == 2 && !(pery && y >= ny - 2)) continue;
    float *rowp = row0 + (long long)(iy == 0 ? 0 : (iy == 1 ? ny : -ny)) * px;
    if (iy > 0) write_chunk(rowp + jl, cs, v, full, room);
    if (perx) {
      if (jl == 0)
        for (int q = 0; q < 3; q++) rowp[q * cs + (nx >> 1)] = v[q].x;
      const int el = (nx >> 1) - 1 - jl;
      if (el >= 0 && el < 4)
        for (int q = 0; q < 3; q++) rowp[q * cs - 1] = f4get(v[q], el);
    }
  }
}

template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY, int NT>
__global__ void __launch_bounds__(NT, NT <= 256 ? 2 : 1) k_sweep_fused(ModelDev m, FusedArgs a) {
  constexpr int PF = Win<TY>::PF, SLOT = Win<TY>::SLOT;
  static_assert((TY + 2) * NPAIR + TY + TY * NPAIR <= 2 * NT, "two task slots per thread must cover a step");
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = smem_align128(smem_dyn);
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
  auto slot_ptr = [&](int p) -> float * { return slots + (size_t)((unsigned)(p - pbeg) % NSL) * SLOT; };
  int last_issued = pbeg - 1;  // meaningful in thread 0 only
  auto issue = [&](int p) {    // thread 0 only
    if (p > pend) return;
    const int lp = p - pbeg;
    last_issued = p;
    if (a.skip_first_load && lp == 0) return;  // test hook: nothing will complete this barrier phase
    unsigned long long *bar = &bars[(unsigned)lp % NSL];
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
      if (plane_exists(p) && !mbar_wait_bounded(&bars[(unsigned)lp % NSL], ((unsigned)lp / NSL) & 1u, a.timeout_ns))
        s_fail = 1;
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
  const TaskSlot ts[2] = {make_slot<TY>(tid), make_slot<TY>(tid + NT)};
  // write-out task: row rr, parity h, chunk of 4 cells q4
  const bool wr_task = tid < TY * 16;
  const int w_rr = tid >> 4, w_h = (tid >> 3) & 1, w_q4 = tid & 7;

  bool ok = wait_plane(z0 - 2) && wait_plane(z0 - 1);
  for (int k = z0 - 1; ok && k <= z1 + 2; k++) {
    ok = wait_plane(k + 1);
    if (!ok) break;
    if (tid == 0) issue(k + 3);
    const bool doA = k <= z1 && plane_exists(k);
    const bool ownA = k >= z0 && k < z1;
    const int kb = k - 2;
    const bool doB = kb >= z0 && kb < z1 && plane_exists(kb);
    float *csA = slot_ptr(k);
    const float *belowA = plane_exists(k - 1) ? slot_ptr(k - 1) : nullptr;
    const float *aboveA = plane_exists(k + 1) ? slot_ptr(k + 1) : nullptr;
    float *csB = slot_ptr(kb);
    const float *belowB = plane_exists(kb - 1) ? slot_ptr(kb - 1) : nullptr;
    const float *aboveB = plane_exists(kb + 1) ? slot_ptr(kb + 1) : nullptr;
    const int zwA = wrapz(k), zwB = wrapz(kb);
    float eB = 0.f;
#pragma unroll 1
    for (int si = 0; si < 2; si++) {
      const TaskSlot t = ts[si];
      float *cs;
      const float *below, *above;
      int y, x, h, jb, zw;
      bool v0, v1, count, meas;
      if (t.type == 0) {  // colour A pair of row y0 - 1 + rr (ring rows only on owned planes)
        if (!doA) continue;
        y = y0 - 1 + t.rr;
        h = (y + k) & 1;
        jb = 4 + 2 * t.p;
        x = x0 + 4 * t.p + h;
        const bool ring_row = t.rr == 0 || t.rr == TY + 1;
        const bool yok = ownA ? (y >= ylo_ring && y <= yhi_ring) : (!ring_row && y < ny);
        v0 = yok && x < nx;
        v1 = yok && x + 2 < nx;
        cs = csA;
        below = belowA;
        above = aboveA;
        zw = zwA;
        count = ownA && !ring_row && y < ny;
        meas = false;
      } else if (t.type == 1) {  // one ring-column site of colour A (owned planes)
        if (!doA || !ownA) continue;
        const int xcol = t.p == 0 ? x0 - 1 : xright;
        y = y0 + 2 * t.rr + ((xcol + y0 + k) & 1);  // (xcol + y + k) even
        const bool valid = (t.p == 0 ? has_left : has_right) && y < y0 + TY && y < ny;
        h = xcol & 1;
        const int jj = (xcol >> 1) - j0 + 4;  // window cell of the site
        jb = jj & ~1;
        x = xcol - 2 * (jj & 1);  // x of the pair's first cell
        v0 = valid && (jj & 1) == 0;
        v1 = valid && (jj & 1) == 1;
        cs = csA;
        below = belowA;
        above = aboveA;
        zw = zwA;
        count = false;
        meas = false;
      } else if (t.type == 2) {  // colour B pair of row y0 + rr of plane k - 2
        if (!doB) continue;
        y = y0 + t.rr;
        h = (y + kb + 1) & 1;
        jb = 4 + 2 * t.p;
        x = x0 + 4 * t.p + h;
        v0 = y < ny && x < nx;
        v1 = y < ny && x + 2 < nx;
        cs = csB;
        below = belowB;
        above = aboveB;
        zw = zwB;
        count = true;
        meas = measure;
      } else {
        continue;
      }
      if (!(v0 | v1)) continue;
      pair_task<POT, GEO, FLIP, PXY, CHIRAL, FIELD, TY>(m, c, cs, below, above, y - y0 + 2, h, jb, x, y, zw, v0, v1,
                                                        count, meas, accepted, eB);
    }
    if (measure) dacc[0] += (double)eB;
    // ---- write-out of plane k - 3 (both colours final): rows x parities x 8 chunks of 4 cells
    const int kw = k - 3;
    if (wr_task && kw >= z0 && kw < z1 && plane_exists(kw)) {
      const float *cw = slot_ptr(kw);
      const int zw = wrapz(kw);
      const int y = y0 + w_rr, h = w_h;
      const int jl = j0 + 4 * w_q4;  // first half-row index of the chunk
      const int xfirst = 2 * jl + h;
      if (y < ny && xfirst < nx) {
        int sid = -1;
        float sz = 0.f;
        if (GEO == GEO_SLAB) sid = slab_surface(zw, nz, sz);
        const int cell = ((w_rr + 2) * 2 + h) * HALF + 4 + 4 * w_q4;
        float4 v[3];
#pragma unroll
        for (int q = 0; q < 3; q++) v[q] = *reinterpret_cast<const float4 *>(cw + q * PF + cell);
        const bool full = xfirst + 6 < nx;
        // half-row (plane zw, row y, parity h) at half index 0, component 0
        float *row0 = a.out + R.off + ((long long)zw * R.py + (y + GY)) * R.px + h * R.hp + GH;
        const long long cs = R.comp;
        write_chunk(row0 + jl, cs, v, full, nx - xfirst);
        // ghost copies (edge chunks only): rows y +- ny along a periodic y, columns along a periodic x
        const int el = (nx >> 1) - 1 - jl;  // element holding half index nx/2 - 1 (nx is even when periodic)
        const bool gx = c.perx && (jl == 0 || (el >= 0 && el < 4));
        const bool gy = c.pery && (y < 2 || y >= ny - 2);
        if (gx || gy) write_ghosts(row0, cs, R.px, v[0], v[1], v[2], full, nx - xfirst, jl, nx, ny, y, c.perx, c.pery);
        if (measure) {
          float f[kPartials];
#pragma unroll
          for (int q = 0; q < kPartials; q++) f[q] = 0.f;
          const bool single = ((h + y + kw) & 1) == 0 && (sid >= 0 || (FIELD && m.field_on));  // colour A terms
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
            if (single) f[0] += single_energy<FIELD>(m, Vec3{vx, vy, vz}, sid, Vec3{0.f, 0.f, sz}, c.elecE);
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
        mbar_wait_bounded(&bars[(unsigned)lp % NSL], ((unsigned)lp / NSL) & 1u, a.timeout_ns);
      }
    }
    __syncthreads();
    return;
  }

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

// Tile configurations: rows per tile, threads per CTA, resident CTAs per SM, the kernel (kind 0 the fused
// two-colour sweep of this file, kind 1 two colour passes, sweep_pass.cuh) and the tile width.
struct FusedCfg {
  int ty, nt, ctas_per_sm, kind, tx;
};
constexpr int kNumCfgs = 5;

// Launch of one potential's kernels (sweep_fused_{ll,ghrl,pear}.cu): dispatch over geometry, flip, periodic x/y,
// chirality, field and tile configuration.
struct FusedLaunch {
  int geo, cfg;
  bool flip, pxy, chiral, field;
  int n_items;
  size_t smem;
  cudaStream_t stream;
  bool prepare = false;  // only set the kernel's shared-memory limit (done once per plan, outside any capture)
};
cudaError_t launch_fused_ll(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);
cudaError_t launch_fused_ghrl(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);
cudaError_t launch_fused_pear(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);
cudaError_t launch_pass_ll(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);
cudaError_t launch_pass_ghrl(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);
cudaError_t launch_pass_pear(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);

template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY, int NT>
cudaError_t launch_fused_one(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  auto k = k_sweep_fused<POT, GEO, FLIP, PXY, CHIRAL, FIELD, TY, NT>;
  if (l.prepare) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem);
  k<<<l.n_items, NT, l.smem, l.stream>>>(m, a);
  return cudaGetLastError();
}

template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD>
cudaError_t launch_fused_cfg(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.cfg == 1) return launch_fused_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 28, 512>(m, a, l);
  return launch_fused_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 14, 256>(m, a, l);
}

template <int POT, bool FLIP, bool CHIRAL, bool FIELD>
cudaError_t launch_fused_gp(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.geo == GEO_SLAB)
    return l.pxy ? launch_fused_cfg<POT, GEO_SLAB, FLIP, true, CHIRAL, FIELD>(m, a, l)
                 : launch_fused_cfg<POT, GEO_SLAB, FLIP, false, CHIRAL, FIELD>(m, a, l);
  return l.pxy ? launch_fused_cfg<POT, GEO_BULK, FLIP, true, CHIRAL, FIELD>(m, a, l)
               : launch_fused_cfg<POT, GEO_BULK, FLIP, false, CHIRAL, FIELD>(m, a, l);
}

}  // namespace mcl
