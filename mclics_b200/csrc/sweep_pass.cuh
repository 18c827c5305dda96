// Colour pass: one colour of the two-colour sweep in one launch, in place, streamed through shared memory by TMA.
//
// In the split-parity layout (common.cuh) the sites of one colour in a row are one contiguous half-row, and every
// neighbour of a colour-c site has colour 1 - c. A pass over colour c therefore reads neighbours that no CTA of the
// same launch writes, and can write its sites back into the buffer it reads: no second buffer, no recomputed ring,
// no halo planes computed twice. A sweep is two passes (colour 0 = x + y + z even, then colour 1), each exactly
// one site update per owned site; the results are bit-identical to the fused kernel's (same draws, same arithmetic,
// same order of colours).
//
// Work item = (replica, TX x TY tile, z segment [z0, z1)). The CTA streams planes z0 - 1 .. z1 through NSLP = 4
// shared-memory slots; each slot is one 5-D TMA box (TX / 2 + 8 half-row cells, 2 parities, TY + 2 rows, 1 plane,
// 3 components) of the split layout, completed on an mbarrier. At step k (plane k) a thread updates the two
// colour-c sites x and x + 2 of one row (adjacent cells of one half-row, paired FP32 lanes, one Philox call),
// reading plane k for the in-plane neighbours and plane k + 1 for the +z neighbours, and stores the pair to global
// memory with the ghost copies of edge sites. The -z neighbours (plane k - 1, the same cells in the parity of the
// step-k sites) are the other-parity cells the thread read at step k - 1, kept in registers, so plane k - 1 leaves
// shared memory before step k: planes k + 2 and k + 3 are in flight while step k runs.
//
// Per-step bookkeeping is kept out of the hot loop:
//  * Thread -> task map by row parity: a warp's tasks lie on rows of one parity (rows r and r + 2 for 64-wide
//    tiles), so the x parity h of its sites is warp-uniform at every plane. The step body is compiled for h = 0 and
//    h = 1 and chosen by a warp-uniform branch; every shared-memory offset of a task is then a register base plus
//    an immediate, and the +x / -x neighbour lanes need no selects.
//  * The x neighbours of a pair are two loads per component: the 8-byte pair of other-parity cells (jb, jb + 1),
//    which is also the next plane's -z neighbour pair and the colour-0 pair the measurement reads, and one scalar
//    cell on the side h selects.
//  * Philox counter, global row pointer and the bounds of both parities are computed once per task and advanced by
//    one addition per plane; ghost copies along x are stored inline by the lanes at the half-row ends.
//  * Uniforms from the draw bits without integer-to-float conversions: for a 21-bit field f, 1 + f 2^-21 is an
//    exact float built by a shift and an OR, so u = (1 + f 2^-21) - 1 is exact and equal to f 2^-21, the value the
//    other kernels compute (flip models keep their 24-bit conversion).
//  * The measurement is a compile-time variant (MEAS: the colour-1 pass of a measured sweep), so the colour-0 pass
//    and unmeasured sweeps hold no accumulators. Every bond has exactly one colour-1 end, so
//    E_total = sum_1 (2 bond + single) + sum_0 single; the colour-1 task adds the raw moments (sum n_a n_b, sum n)
//    of its two updated sites and of the two colour-0 sites of the same cells in the other half-row (final since
//    the colour-0 pass), summed in FP32 over the thread's work item (at most 4 sites per plane of its segment),
//    then in FP64 over threads, CTAs and the grid; each thread turns its moments into
//    sum Q = 1.5 sum n_a n_b - 0.5 delta_ab N.
//
// Every wait on a TMA barrier is bounded by %globaltimer; on timeout the CTA sets the error word, waits (bounded)
// for its copies in flight and returns, and the host reports MCL_ERR_CUDA.
#pragma once
#include <type_traits>

#include "sweep_fused.cuh"

namespace mcl {

constexpr int NSLP = 4;

// Plane window of a TX x TY tile: per row and parity TX / 2 + 8 half-row cells (the tile's TX / 2 and 4 on each
// side, 16-byte aligned), TY + 2 rows, 3 components.
template <int TY, int TX>
struct PassWin {
  static constexpr int HW = TX / 2 + 8, RWX = 2 * HW, NP = TX / 4;  // cells per half-row, per row; pairs per row
  static constexpr int H = TY + 2, PF = RWX * H, SLOT = (3 * PF + 31) / 32 * 32;
};

// Ghost copies of the updated pair (elements e = 0, 1 at half indices jl, jl + 1 of the half-row `row0` of parity
// h, component 0): along a periodic y the pair again at rows y + ny (y < 2) and y - ny (y >= ny - 2); along a
// periodic x, on each of those rows, half index nx / 2 for half index 0 and half index -1 for nx / 2 - 1.
static __device__ __noinline__ void pass_ghosts(float *row0, long long cs, int px, float v0x, float v0y, float v0z,
                                                float v1x, float v1y, float v1z, bool has1, int jl, int nx, int ny,
                                                int y, bool perx, bool pery) {
  const float v[2][3] = {{v0x, v0y, v0z}, {v1x, v1y, v1z}};
  for (int iy = 0; iy < 3; iy++) {
    if (iy == 1 && !(pery && y < 2)) continue;
    if (iy == 2 && !(pery && y >= ny - 2)) continue;
    float *rowp = row0 + (long long)(iy == 0 ? 0 : (iy == 1 ? ny : -ny)) * px;
    for (int e = 0; e < 2; e++) {
      if (e == 1 && !has1) break;
      const int j = jl + e;
      if (iy > 0)
        for (int q = 0; q < 3; q++) rowp[q * cs + j] = v[e][q];
      if (perx && j == 0)
        for (int q = 0; q < 3; q++) rowp[q * cs + (nx >> 1)] = v[e][q];
      if (perx && j == (nx >> 1) - 1)
        for (int q = 0; q < 3; q++) rowp[q * cs - 1] = v[e][q];
    }
  }
}

// Raw moments of two pairs of sites (lanes paired): m[0..5] = sum v_a v_b (xx, xy, xz, yy, yz, zz), m[6..8] = sum v.
// Q and sum n follow per thread at the end: sum q_ab = 1.5 sum v_a v_b - 0.5 delta_ab (sites).
__device__ __forceinline__ void pair_moments(float2 (&m)[9], const float2 (&u)[3], const float2 (&v)[3]) {
  m[0] = __ffma2_rn(v[0], v[0], __fmul2_rn(u[0], u[0]));
  m[1] = __ffma2_rn(v[0], v[1], __fmul2_rn(u[0], u[1]));
  m[2] = __ffma2_rn(v[0], v[2], __fmul2_rn(u[0], u[2]));
  m[3] = __ffma2_rn(v[1], v[1], __fmul2_rn(u[1], u[1]));
  m[4] = __ffma2_rn(v[1], v[2], __fmul2_rn(u[1], u[2]));
  m[5] = __ffma2_rn(v[2], v[2], __fmul2_rn(u[2], u[2]));
  m[6] = __fadd2_rn(u[0], v[0]);
  m[7] = __fadd2_rn(u[1], v[1]);
  m[8] = __fadd2_rn(u[2], v[2]);
}

// Warp w of the CTA covers rows of parity w & 1: rows pc + 2 (RPW (w >> 1) + lane / NP), pair lane % NP.
template <int TY, int TX, int NT>
struct TaskMap {
  static constexpr int NP = TX / 4;   // pairs per row
  static constexpr int RPW = 32 / NP; // rows per warp
  static_assert(NT == TY * NP, "one pair task per thread and plane");
  static_assert(32 % NP == 0 && TY % (2 * RPW) == 0, "a warp's rows share one parity");
  __device__ __forceinline__ static int row(int tid) {
    const int w = tid >> 5, l = tid & 31;
    return (w & 1) + 2 * (RPW * (w >> 1) + l / NP);
  }
  __device__ __forceinline__ static int pair(int tid) { return tid & (NP - 1); }
};

// Lane values of a pair draw (one Philox block for sites x and x + 2, non-flip models), bit-identical to
// lane_draw(pair_half(out, 0), pair_half(out, 1), false).
__device__ __forceinline__ float unit21_bits(uint32_t bits_shifted, uint32_t exponent) {
  return __uint_as_float(exponent | (bits_shifted & 0x7FFFFCu));
}
__device__ __forceinline__ LaneDraw<float2> pair_draw_lanes(const U4 &o) {
  LaneDraw<float2> r;
  // u1 (angle field, bits 0..20 of lo): 2 u1 - 1 is used; keep u1 itself exact as (1 + f 2^-21) - 1
  r.u1 = __fadd2_rn(make_float2(unit21_bits(o.x << 2, 0x3F800000u), unit21_bits(o.z << 2, 0x3F800000u)),
                    make_float2(-1.f, -1.f));
  // u3 (acceptance field, bits 10..30 of hi)
  r.u3 = __fadd2_rn(make_float2(unit21_bits(o.y >> 8, 0x3F800000u), unit21_bits(o.w >> 8, 0x3F800000u)),
                    make_float2(-1.f, -1.f));
  r.u4 = make_float2(0.f, 0.f);
  // axis field: bits 21..41 of the 64-bit half (lo, hi)
  const uint32_t f0 = __funnelshift_r(o.x, o.y, 21) & 0x1FFFFFu, f1 = __funnelshift_r(o.z, o.w, 21) & 0x1FFFFFu;
  r.w0 = make_float2(f0 < 698352u ? 1.f : 0.f, f1 < 698352u ? 1.f : 0.f);
  r.w2 = make_float2(f0 >= 1396704u ? 1.f : 0.f, f1 >= 1396704u ? 1.f : 0.f);
  r.w1 = make_float2(1.f - r.w0.x - r.w2.x, 1.f - r.w0.y - r.w2.y);
  return r;
}

// An 8-byte shared-memory load the compiler may not merge with an earlier load of the same address (a merge would
// keep the value in registers across the code between them).
__device__ __forceinline__ float2 lds_f2(const float *p) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(smem_u32(p)));
  return v;
}

template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY, int NT, int MINB, int TX, bool MEAS>
__global__ void __launch_bounds__(NT, MINB) k_sweep_pass(ModelDev m, FusedArgs a) {
  using W = PassWin<TY, TX>;
  using MP = TaskMap<TY, TX, NT>;
  constexpr int PF = W::PF, SLOT = W::SLOT, HALF = W::HW, RW = W::RWX;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *smem_raw = smem_align128(smem_dyn);
  float *slots = reinterpret_cast<float *>(smem_raw);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + (size_t)NSLP * SLOT * 4);
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
  const int colour = a.colour;
  constexpr bool measure = MEAS;  // the colour-1 pass with the observables (a.measure != 0, colour 1)
  const unsigned long long seed = R.seed, sweep = *a.sweep_ctr;
  const float T = S.T, invT = 1.f / S.T, av = S.ang_var, elecE = S.elecE;
  constexpr unsigned box_bytes = 3u * PF * 4u;

  if (tid == 0) {
    s_fail = 0;
    for (int q = 0; q < NSLP; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
  }
  __syncthreads();

  // Planes z0 - 1 .. z1 stream through the NSLP slots (plane p in slot (p - pbeg) % NSLP).
  const int pbeg = z0 - 1, pend = z1;
  const int zoff = R.zoff, nzg = R.nzg;
  const int pz_lo = R.zslab ? -zoff : 0, pz_hi = R.zslab ? nzg - zoff : nz;
  auto plane_exists = [&](int p) { return perz || (p >= pz_lo && p < pz_hi); };
  auto wrapz = [&](int p) { return p < 0 ? p + nz : (p >= nz ? p - nz : p); };
  int last_issued = pbeg - 1;  // thread 0 only
  auto issue = [&](int p) {    // thread 0 only
    if (p > pend) return;
    const int lp = p - pbeg;
    last_issued = p;
    if (a.skip_first_load && lp == 0) return;  // test hook: nothing will complete this barrier phase
    unsigned long long *bar = &bars[lp & (NSLP - 1)];
    if (!plane_exists(p)) {
      mbar_arrive(bar);
      return;
    }
    mbar_expect_tx(bar, box_bytes);
    tma_load_plane(slots + (lp & (NSLP - 1)) * SLOT, map, j0, y0 - 1 + GY, wrapz(p), bar);
  };
  // Bounded wait for plane p (every thread), then the CTA barrier that also frees the slot of plane p - 2.
  auto wait_plane = [&](int p) -> bool {
    if (p <= pend && plane_exists(p)) {
      const int lp = p - pbeg;
      if (!mbar_wait_bounded(&bars[lp & (NSLP - 1)], (unsigned)(lp >> 2) & 1u, a.timeout_ns)) s_fail = 1;
    }
    __syncthreads();
    return s_fail == 0;
  };
  if (tid == 0)
    for (int p = pbeg; p <= pbeg + 3; p++) issue(p);

  // ---- the task of this thread --------------------------------------------------------------------------------
  const int r = MP::row(tid), pr = MP::pair(tid);
  const int y = y0 + r;
  const bool live = y < ny;
  const int pc = r & 1;                           // warp-uniform
  const int jb = 4 + 2 * pr;                      // window cell of the pair's first site
  const int jl = j0 + 2 * pr;                     // its half-row index
  const int rowb = (r + 1) * 2 * HALF + jb;       // window offset of parity 0, cell jb, of row y
  const int xb = x0 + 4 * pr;                     // site x of the pair is xb + h
  // bounds of both parities: lane 0 (x = xb + h), lane 1 (x + 2), colour-0 sites of the other parity (xb + 1 - h)
  const bool v0h[2] = {xb < nx, xb + 1 < nx}, v1h[2] = {xb + 2 < nx, xb + 3 < nx};
  const long long cs = R.comp;
  float *grow = a.out + R.off + ((long long)z0 * R.py + (y + GY)) * R.px + GH + jl;  // plane z0, parity 0
  const long long gplane = (long long)R.py * R.px;
  const int hp = R.hp;
  const uint32_t nxny = (uint32_t)nx * (uint32_t)ny;
  uint32_t ctr = (uint32_t)xb + (uint32_t)nx * ((uint32_t)y + (uint32_t)ny * (uint32_t)(z0 + zoff));  // plane z0, h = 0
  const bool perx = R.periodic[0], pery = R.periodic[1];
  // Ghost copies written with the pair. Rows y < 2 and y >= ny - 2 of a periodic y (all of their copies, x ones
  // included) go through pass_ghosts; on other rows a periodic x needs at most the copy of the half-row's first site
  // at half index nx / 2 (jl == 0) and of its last site at -1 (element 0 when jl == nx / 2 - 1, element 1 when
  // jl + 1 == nx / 2 - 1), stored inline.
  const bool yghost = pery && (y < 2 || y >= ny - 2);
  const bool xg_first = perx && jl == 0, xg_last0 = perx && jl == (nx >> 1) - 1,
             xg_last1 = perx && jl + 1 == (nx >> 1) - 1;
  const int dx_first = nx >> 1, dx_last = -1 - jl;  // offsets from the pair's first cell
  // neighbour weights of free x / y edges (PXY: all present)
  float2 wxp[2], wxm[2], wyp, wym;
  if (!PXY) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int x = xb + h;
      wxp[h] = make_float2((perx || x + 1 < nx) ? 1.f : 0.f, (perx || x + 3 < nx) ? 1.f : 0.f);
      wxm[h] = make_float2((perx || x - 1 >= 0) ? 1.f : 0.f, 1.f);
    }
    const float a_ = (pery || y + 1 < ny) ? 1.f : 0.f, b_ = (pery || y - 1 >= 0) ? 1.f : 0.f;
    wyp = make_float2(a_, a_);
    wym = make_float2(b_, b_);
  }

  unsigned accepted = 0;
  int n_meas = 0;
  // The thread's sums over its work item (at most 4 sites per plane of its z segment) in FP32: ten FP32
  // registers instead of ten FP64 pairs keep the measured pass at the unmeasured pass's occupancy. The threads' sums
  // are then added in FP64 (warp shuffles, the CTA, the grid).
  float facc[kPartials];
#pragma unroll
  for (int q = 0; q < kPartials; q++) facc[q] = 0.f;
  auto add_step = [&](const float2 (&f)[kPartials]) {
#pragma unroll
    for (int q = 0; q < kPartials; q++) facc[q] += f[q].x + f[q].y;
  };

  bool ok = wait_plane(z0 - 1) && wait_plane(z0);
  // -z neighbours of the first plane: plane z0 - 1, the parity of this task's sites in plane z0
  float2 pd[3];
#pragma unroll
  for (int q = 0; q < 3; q++) pd[q] = make_float2(0.f, 0.f);
  {
    const int h = (colour + y0 + pc + z0 + zoff) & 1;
    if (ok && live && plane_exists(z0 - 1)) {
      const float *src = slots + ((z0 - 1 - pbeg) & (NSLP - 1)) * SLOT + rowb + h * HALF;
#pragma unroll
      for (int q = 0; q < 3; q++) pd[q] = *reinterpret_cast<const float2 *>(src + q * PF);
    }
  }

  // single-site terms: none in a bulk lattice without a field; a slab's step body keeps them on every plane (a
  // second, surface-only variant of the body pushes the 80-register kernels into spilling)
  constexpr bool kNever = GEO == GEO_BULK && !FIELD, kAlways = FIELD || GEO == GEO_SLAB;
  for (int k = z0; ok && k < z1; k++) {
    ok = wait_plane(k + 1);
    if (!ok) break;
    if (tid == 0) issue(k + 3);
    if (live) {
      const int h = (colour + y0 + pc + k + zoff) & 1;  // warp-uniform
      const float *sk = slots + ((k - pbeg) & (NSLP - 1)) * SLOT + rowb;
      const bool has_above = plane_exists(k + 1), has_below = plane_exists(k - 1);
      const float *sa = has_above ? slots + ((k + 1 - pbeg) & (NSLP - 1)) * SLOT + rowb : sk;
      const int zg = k + zoff;
      int sid = -1;
      float sz = 0.f;
      if (!kNever && GEO == GEO_SLAB) sid = slab_surface(zg, nzg, sz);
      const bool single_terms = kNever ? false : (kAlways ? true : (zg == 0 || zg == nzg - 1));
      auto body = [&](auto h_tag, auto single_tag) {
        constexpr int H = decltype(h_tag)::value;
        constexpr bool SINGLE = decltype(single_tag)::value;
        const float *own = sk + H * HALF;
        const float *oc = sk + (H ^ 1) * HALF;  // other-parity cells jb, jb + 1
        const float *zu = sa + H * HALF;
        float2 pn[3];
#pragma unroll
        for (int q = 0; q < 3; q++) pn[q] = *reinterpret_cast<const float2 *>(oc + q * PF);
        // colour-0 sites of the other parity in the same cells (measured by the colour-1 pass): xb + (H ^ 1) + 2 e
        const bool c0 = xb + (H ^ 1) < nx, c1 = xb + (H ^ 1) + 2 < nx;
        const Vec3 sn{0.f, 0.f, sz};
        // moments and single-site energies of the colour-0 lanes that exist (va), added to the group sums
        auto measure_colour0 = [&](float2 &eb, float2 (&va)[3]) {
          if (SINGLE) {
            const float2 s0 = single_energy<FIELD>(m, V3<float2>{pn[0], pn[1], pn[2]}, sid, sn, elecE);
            eb.x += c0 ? s0.x : 0.f;
            eb.y += c1 ? s0.y : 0.f;
          }
#pragma unroll
          for (int q = 0; q < 3; q++) va[q] = make_float2(c0 ? pn[q].x : 0.f, c1 ? pn[q].y : 0.f);
          n_meas += (int)c0 + (int)c1;
        };
        if (!v0h[H]) {  // the pair lies beyond the ragged right edge: only carry the -z neighbours
          if (measure && c0) {  // odd nx (free x): the colour-0 site at nx - 1 is still measured here
            float2 eb = make_float2(0.f, 0.f), va[3];
            measure_colour0(eb, va);
            const float2 f[kPartials] = {eb,
                                         __fmul2_rn(va[0], va[0]),
                                         __fmul2_rn(va[0], va[1]),
                                         __fmul2_rn(va[0], va[2]),
                                         __fmul2_rn(va[1], va[1]),
                                         __fmul2_rn(va[1], va[2]),
                                         __fmul2_rn(va[2], va[2]),
                                         va[0],
                                         va[1],
                                         va[2]};
            add_step(f);
          }
#pragma unroll
          for (int q = 0; q < 3; q++) pd[q] = pn[q];
          return;
        }
        float2 o[3], yu[3], yd[3], pu[3];
        float sx[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
          o[q] = *reinterpret_cast<const float2 *>(own + q * PF);
          yu[q] = *reinterpret_cast<const float2 *>(own + q * PF + RW);
          yd[q] = *reinterpret_cast<const float2 *>(own + q * PF - RW);
          pu[q] = *reinterpret_cast<const float2 *>(zu + q * PF);
          sx[q] = H == 0 ? oc[q * PF - 1] : oc[q * PF + 2];
        }
        LaneDraw<float2> ld;
        if (FLIP) {
          const U4 u0 = site_draws(seed, sweep, ctr + H, 0), u1 = site_draws(seed, sweep, ctr + H + 2, 0);
          ld = lane_draw(Draw{u0.x >> 8, u0.y >> 8, u0.z >> 8, u0.w >> 8},
                         Draw{u1.x >> 8, u1.y >> 8, u1.z >> 8, u1.w >> 8}, true);
        } else {
          ld = pair_draw_lanes(site_draws(seed, sweep, ctr + H, 0));
        }
        const V3<float2> n{o[0], o[1], o[2]};
        // +x / -x neighbour lanes: h = 0: +x = (jb, jb + 1), -x = (jb - 1, jb); h = 1: +x = (jb + 1, jb + 2),
        // -x = (jb, jb + 1)
        V3<float2> nbx_p, nbx_m;
        if (H == 0) {
          nbx_p = V3<float2>{pn[0], pn[1], pn[2]};
          nbx_m = V3<float2>{make_float2(sx[0], pn[0].x), make_float2(sx[1], pn[1].x), make_float2(sx[2], pn[2].x)};
        } else {
          nbx_p = V3<float2>{make_float2(pn[0].y, sx[0]), make_float2(pn[1].y, sx[1]), make_float2(pn[2].y, sx[2])};
          nbx_m = V3<float2>{pn[0], pn[1], pn[2]};
        }
        const V3<float2> nb[6] = {nbx_p, nbx_m, V3<float2>{yu[0], yu[1], yu[2]}, V3<float2>{yd[0], yd[1], yd[2]},
                                  V3<float2>{pu[0], pu[1], pu[2]}, V3<float2>{pd[0], pd[1], pd[2]}};
        float2 w[6];
        if (PXY) {
          w[0] = w[1] = w[2] = w[3] = make_float2(1.f, 1.f);
        } else {
          w[0] = wxp[H];
          w[1] = wxm[H];
          w[2] = wyp;
          w[3] = wym;
        }
        const float wzu = has_above ? 1.f : 0.f, wzd = has_below ? 1.f : 0.f;
        w[4] = make_float2(wzu, wzu);
        w[5] = make_float2(wzd, wzd);
        const SiteResultT<float2> res =
            site_update<POT, FLIP, PXY, CHIRAL, FIELD, float2, SINGLE>(m, n, nb, w, sid, sn, elecE, ld, av, T, invT);
        // the other-parity pair again (not kept live across the physics): the colour-0 sites measured below and
        // the next plane's -z neighbours
#pragma unroll
        for (int q = 0; q < 3; q++) pn[q] = lds_f2(oc + q * PF);
        const bool v1 = v1h[H];
        const float2 fin[3] = {make_float2(res.n.x.x, v1 ? res.n.x.y : o[0].y),
                               make_float2(res.n.y.x, v1 ? res.n.y.y : o[1].y),
                               make_float2(res.n.z.x, v1 ? res.n.z.y : o[2].y)};
        float *g = grow + H * hp;
        if (v1) {
#pragma unroll
          for (int q = 0; q < 3; q++) *reinterpret_cast<float2 *>(g + q * cs) = fin[q];
        } else {
#pragma unroll
          for (int q = 0; q < 3; q++) g[q * cs] = fin[q].x;
        }
        if (yghost) {
          pass_ghosts(g - jl, cs, R.px, fin[0].x, fin[1].x, fin[2].x, fin[0].y, fin[1].y, fin[2].y, v1, jl, nx, ny, y,
                      perx, pery);
        } else {
          if (xg_first) {
#pragma unroll
            for (int q = 0; q < 3; q++) g[q * cs + dx_first] = fin[q].x;
          }
          if (xg_last0 || xg_last1) {
#pragma unroll
            for (int q = 0; q < 3; q++) g[q * cs + dx_last] = xg_last0 ? fin[q].x : fin[q].y;
          }
        }
        accepted += (res.rot.x ? 1u : 0u) + (v1 && res.rot.y ? 1u : 0u);
        if (measure) {
          // colour-1 sites (fin) with 2 bond + single, and the colour-0 sites of the other parity (pn) with single
          float2 eb = __ffma2_rn(make_float2(2.f, 2.f), res.bond, res.single);
          if (!v1) eb.y = 0.f;
          float2 vb[3], va[3];
          measure_colour0(eb, va);
#pragma unroll
          for (int q = 0; q < 3; q++) vb[q] = make_float2(fin[q].x, v1 ? fin[q].y : 0.f);
          n_meas += 1 + (int)v1;
          float2 f[kPartials];
          f[0] = eb;
          pair_moments(reinterpret_cast<float2(&)[9]>(f[1]), vb, va);
          add_step(f);
        }
#pragma unroll
        for (int q = 0; q < 3; q++) pd[q] = pn[q];
      };
      if (h) {
        if (single_terms) body(std::integral_constant<int, 1>{}, std::true_type{});
        else body(std::integral_constant<int, 1>{}, std::false_type{});
      } else {
        if (single_terms) body(std::integral_constant<int, 0>{}, std::true_type{});
        else body(std::integral_constant<int, 0>{}, std::false_type{});
      }
    }
    grow += gplane;
    ctr += nxny;
  }

  if (!ok) {
    if (tid == 0) {
      atomicOr(a.err, 1u);
      for (int q = max(pbeg, last_issued - NSLP + 1); q <= last_issued; q++) {
        if (!plane_exists(q) || (a.skip_first_load && q == pbeg)) continue;
        const int lp = q - pbeg;
        mbar_wait_bounded(&bars[lp & (NSLP - 1)], (unsigned)(lp >> 2) & 1u, a.timeout_ns);
      }
    }
    __syncthreads();
    return;
  }

  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&a.st[it.rep].acc, (unsigned long long)wsum);
  if (measure) {
    // raw moments -> sum of q = 1.5 v_a v_b - 0.5 delta_ab (partials 1..6: xx, xy, xz, yy, yz, zz)
    double dsum[kPartials];
#pragma unroll
    for (int q = 0; q < kPartials; q++) dsum[q] = (double)facc[q];
#pragma unroll
    for (int q = 1; q <= 6; q++) dsum[q] *= 1.5;
    dsum[1] -= 0.5 * n_meas;
    dsum[4] -= 0.5 * n_meas;
    dsum[6] -= 0.5 * n_meas;
    __shared__ double red[NT / 32][kPartials];
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < kPartials; q++) {
      double v = dsum[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (tid < kPartials) {
      double v = 0.0;
      for (int w = 0; w < NT / 32; w++) v += red[w][tid];
      a.partials[(long long)blockIdx.x * kPartials + tid] = v;
    }
  }
}

// One tile configuration: the unmeasured passes and the measured one (the colour-1 pass of a measured sweep).
template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY, int NT, int MINB, int TX>
cudaError_t launch_pass_one(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  auto k0 = k_sweep_pass<POT, GEO, FLIP, PXY, CHIRAL, FIELD, TY, NT, MINB, TX, false>;
  auto k1 = k_sweep_pass<POT, GEO, FLIP, PXY, CHIRAL, FIELD, TY, NT, MINB, TX, true>;
  if (l.prepare) {
    const cudaError_t e = cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem);
    return e != cudaSuccess ? e : cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem);
  }
  if (a.measure != 0 && a.colour == 1)
    k1<<<l.n_items, NT, l.smem, l.stream>>>(m, a);
  else
    k0<<<l.n_items, NT, l.smem, l.stream>>>(m, a);
  return cudaGetLastError();
}

// Colour-pass tile configurations (numbering continues the fused kernel's): 2: 64 x 16, 256 threads, 3 CTAs/SM;
// 3: 64 x 16, 256 threads, 2 CTAs/SM (flip models, whose second trial needs the registers); 4: 32 x 16, 128 threads,
// 5 CTAs/SM (narrow lattices waste less of a tile).
template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD>
cudaError_t launch_pass_cfg(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.cfg == 3) return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 256, 2, 64>(m, a, l);
  if (l.cfg == 4) return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 128, 5, 32>(m, a, l);
  return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 256, 3, 64>(m, a, l);
}

template <int POT, bool FLIP, bool CHIRAL, bool FIELD>
cudaError_t launch_pass_gp(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.geo == GEO_SLAB)
    return l.pxy ? launch_pass_cfg<POT, GEO_SLAB, FLIP, true, CHIRAL, FIELD>(m, a, l)
                 : launch_pass_cfg<POT, GEO_SLAB, FLIP, false, CHIRAL, FIELD>(m, a, l);
  return l.pxy ? launch_pass_cfg<POT, GEO_BULK, FLIP, true, CHIRAL, FIELD>(m, a, l)
               : launch_pass_cfg<POT, GEO_BULK, FLIP, false, CHIRAL, FIELD>(m, a, l);
}

}  // namespace mcl
