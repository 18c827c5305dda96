// Colour pass: one colour of the two-colour sweep in one launch, in place, streamed through shared memory by TMA.
//
// In the split-parity layout (common.cuh) the sites of one colour in a row are one contiguous half-row, and every
// neighbour of a colour-c site has colour 1 - c. A pass over colour c therefore reads neighbours that no CTA of the
// same launch writes, and can write its sites back into the buffer it reads: no second buffer, no recomputed ring,
// no halo planes computed twice. A sweep is two passes (colour 0 = x + y + z even, then colour 1), each exactly
// one site update per owned site; the results are bit-identical to the fused kernel's (same draws, same arithmetic,
// same order of colours).
//
// Work item = (replica, 64 x TY tile, z segment [z0, z1)). The CTA streams planes z0 - 1 .. z1 through NSLP = 4
// shared-memory slots; each slot is one 5-D TMA box (40 half-row cells, 2 parities, TY + 2 rows, 1 plane, 3
// components) of the split layout, completed on an mbarrier. At step k (plane k) thread (row r, pair p) updates the
// two colour-c sites x and x + 2 of row y0 + r (adjacent cells of one half-row, paired FP32 lanes, one Philox call),
// reading plane k for the in-plane neighbours and plane k + 1 for the +z neighbours, and stores the pair to global
// memory with the ghost copies of edge sites. The -z neighbours (plane k - 1, the same cells in the parity of the
// step-k sites) are the other-parity cells the thread read at step k - 1, kept in registers, so plane k - 1 leaves
// shared memory before step k: planes k + 2 and k + 3 are in flight while step k runs.
//
// Measurement (colour-1 pass): every bond has exactly one colour-1 end, so E_total = sum_1 (2 bond + single) +
// sum_0 single; the colour-1 task also adds the raw moments (sum n_a n_b, sum n) of its two updated sites and of
// the two colour-0 sites of the same cells in the other half-row (final since the colour-0 pass), summed in FP32
// per task and step, then in FP64; each thread turns its moments into sum Q = 1.5 sum n_a n_b - 0.5 delta_ab N.
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

template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY, int NT, int MINB, int TPT,
          int TX>
__global__ void __launch_bounds__(NT, MINB) k_sweep_pass(ModelDev m, FusedArgs a) {
  using W = PassWin<TY, TX>;
  constexpr int PF = W::PF, SLOT = W::SLOT, HALF = W::HW, RW = W::RWX, NP = W::NP;
  static_assert(NT * TPT == TY * NP, "TPT pair tasks per thread and plane");
  static_assert(TPT == 1 || (TY / TPT) % 2 == 0, "a thread's rows must share their parity pattern");
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
  const bool measure = a.measure != 0 && colour == 1;
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
    for (int q = 0; q < NSLP; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
  }
  __syncthreads();

  // Plane p (local index lp = p - pbeg) lives in slot lp % NSLP; every use of a slot completes one barrier phase.
  // A z-slab's halo planes (local 0 and nz - 1) exist unless they lie beyond a free global boundary; its work items
  // cover the owned planes only, so no local plane index wraps. zoff = 0, nzg = nz otherwise.
  const int pbeg = z0 - 1, pend = z1;
  const int zoff = R.zoff, nzg = R.nzg;
  const int pz_lo = R.zslab ? -zoff : 0, pz_hi = R.zslab ? nzg - zoff : nz;
  auto plane_exists = [&](int p) { return perz || (p >= pz_lo && p < pz_hi); };
  auto wrapz = [&](int p) { return p < 0 ? p + nz : (p >= nz ? p - nz : p); };
  auto slot_ptr = [&](int p) -> float * { return slots + (size_t)((unsigned)(p - pbeg) % NSLP) * SLOT; };
  int last_issued = pbeg - 1;  // meaningful in thread 0 only
  auto issue = [&](int p) {    // thread 0 only
    if (p > pend) return;
    const int lp = p - pbeg;
    last_issued = p;
    if (a.skip_first_load && lp == 0) return;  // test hook: nothing will complete this barrier phase
    unsigned long long *bar = &bars[(unsigned)lp % NSLP];
    if (!plane_exists(p)) {  // no copy: complete the slot's phase anyway
      mbar_arrive(bar);
      return;
    }
    mbar_expect_tx(bar, box_bytes);
    tma_load_plane(slot_ptr(p), map, j0, y0 - 1 + GY, wrapz(p), bar);  // box rows y0 - 1 .. y0 + TY
  };
  int waited = pbeg - 1;  // uniform: highest plane waited for successfully
  auto wait_plane = [&](int p) -> bool {
    if (p <= pend && p > waited) {
      const int lp = p - pbeg;
      if (plane_exists(p) && !mbar_wait_bounded(&bars[(unsigned)lp % NSLP], ((unsigned)lp / NSLP) & 1u, a.timeout_ns))
        s_fail = 1;
    }
    __syncthreads();
    if (s_fail) return false;
    if (p > waited) waited = p;
    return true;
  };
  // Slot reuse: step k reads planes k and k + 1 only (the -z neighbours of a task are the other-parity cells the
  // same thread read at step k - 1, carried in registers); plane k + 3 goes into the slot of plane k - 1, whose last
  // reader was step k - 1 (the barrier at the start of step k separates them). Two planes are in flight meanwhile.
  if (tid == 0)
    for (int p = pbeg; p <= pbeg + 3; p++) issue(p);

  unsigned accepted = 0;
  int n_meas = 0;  // sites whose raw moments this thread summed
  double dacc[kPartials];
#pragma unroll
  for (int q = 0; q < kPartials; q++) dacc[q] = 0.0;

  // tasks of this thread: pair p of rows rr[t] = r0 + t TY / TPT (same parity pattern: TY / TPT is even)
  const int r0 = tid / NP, p = tid % NP;
  int rr[TPT];
  bool live[TPT];
#pragma unroll
  for (int t = 0; t < TPT; t++) {
    rr[t] = r0 + t * (TY / TPT);
    live[t] = y0 + rr[t] < ny;
  }
  const int jb = 4 + 2 * p;   // window cell of the pair's first site
  const int jl = j0 + 2 * p;  // half index of the pair's first site
  const long long cs = R.comp;

  bool ok = wait_plane(z0 - 1) && wait_plane(z0);
  // -z neighbours of the first step: plane z0 - 1, row y, the parity of this thread's sites in plane z0
  float2 pd[TPT][3];
#pragma unroll
  for (int t = 0; t < TPT; t++) {
#pragma unroll
    for (int q = 0; q < 3; q++) pd[t][q] = make_float2(0.f, 0.f);
    if (ok && live[t] && plane_exists(z0 - 1)) {
      const float *q0 = slot_ptr(z0 - 1) + ((rr[t] + 1) * 2 + ((colour + y0 + rr[t] + z0 + zoff) & 1)) * HALF + jb;
#pragma unroll
      for (int q = 0; q < 3; q++) pd[t][q] = *reinterpret_cast<const float2 *>(q0 + q * PF);
    }
  }
  for (int k = z0; ok && k < z1; k++) {
    ok = wait_plane(k + 1);
    if (!ok) break;
    if (tid == 0) issue(k + 3);
    if (!live[0]) continue;  // rows grow with t: a dead first row has no live rows after it
    const int h = (colour + y0 + r0 + k + zoff) & 1;  // colours follow global planes (zoff: z-slab offset)
    const int x = x0 + 4 * p + h;
    const bool v0 = x < nx, v1 = x + 2 < nx;
    const float *cs_k = slot_ptr(k);
    if (!v0) {  // the other-parity cells are still the next step's -z neighbours
#pragma unroll
      for (int t = 0; t < TPT; t++)
        if (live[t]) {
          const float *src = cs_k + ((rr[t] + 1) * 2 + (h ^ 1)) * HALF + jb;
#pragma unroll
          for (int q = 0; q < 3; q++) pd[t][q] = *reinterpret_cast<const float2 *>(src + q * PF);
        }
      continue;
    }
    // Surface planes and field models take the general path; everything else has no single-site term (bulk
    // without a field: never). With one task per thread a slab runs the general path on every plane (a second copy
    // of the update costs registers that the 3-CTA configuration does not have; the runtime surface test then
    // makes the site terms zero).
    constexpr bool kNever = GEO == GEO_BULK && !FIELD, kAlways = FIELD || (GEO == GEO_SLAB && TPT == 1);
    const bool single_terms = kNever ? false : (kAlways ? true : (k + zoff == 0 || k + zoff == nzg - 1));
    auto step = [&](auto single_tag) {
      constexpr bool SINGLE = decltype(single_tag)::value;
      const bool has_below = plane_exists(k - 1);
      const float *above = plane_exists(k + 1) ? slot_ptr(k + 1) : nullptr;
      const int zw = k;         // computed planes lie inside the local lattice
      const int zg = k + zoff;  // and this is their global index (draws, surfaces)
      int sid = -1;
      float sz = 0.f;
      if (SINGLE && GEO == GEO_SLAB) sid = slab_surface(zg, nzg, sz);
      const Vec3 sn{0.f, 0.f, sz};
      float2 o[TPT][3];
      SiteResultT<float2> res[TPT];
#pragma unroll
      for (int t = 0; t < TPT; t++) {
        const int y = y0 + rr[t];
        const float *own = cs_k + ((rr[t] + 1) * 2 + h) * HALF + jb;
        const float *oth = cs_k + ((rr[t] + 1) * 2 + (h ^ 1)) * HALF + jb - 1 + h;  // 3 consecutive cells
        const float *zu = above ? above + ((rr[t] + 1) * 2 + h) * HALF + jb : own;
        float2 yu[3], yd[3], pu[3];
        float xa[3], xb[3], xc[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
          o[t][q] = *reinterpret_cast<const float2 *>(own + q * PF);
          yu[q] = *reinterpret_cast<const float2 *>(own + q * PF + RW);
          yd[q] = *reinterpret_cast<const float2 *>(own + q * PF - RW);
          pu[q] = *reinterpret_cast<const float2 *>(zu + q * PF);
          xa[q] = oth[q * PF];
          xb[q] = oth[q * PF + 1];
          xc[q] = oth[q * PF + 2];
        }
        Draw d0, d1;
        if (FLIP) {
          d0 = site_draw(c.seed, c.sweep, x, y, zg, nx, ny, true);
          d1 = site_draw(c.seed, c.sweep, x + 2, y, zg, nx, ny, true);
        } else {  // one Philox call serves both sites (x & ~2 is shared: x % 4 = h)
          const U4 out = site_draws(c.seed, c.sweep, pair_counter(x, y, zg, nx, ny), 0);
          d0 = pair_half(out, 0u);
          d1 = pair_half(out, 1u);
        }
        const LaneDraw<float2> ld = lane_draw(d0, d1, FLIP);
        const V3<float2> n{o[t][0], o[t][1], o[t][2]};
        const V3<float2> nb[6] = {
            V3<float2>{make_float2(xb[0], xc[0]), make_float2(xb[1], xc[1]), make_float2(xb[2], xc[2])},  // +x
            V3<float2>{make_float2(xa[0], xb[0]), make_float2(xa[1], xb[1]), make_float2(xa[2], xb[2])},  // -x
            V3<float2>{yu[0], yu[1], yu[2]},
            V3<float2>{yd[0], yd[1], yd[2]},
            V3<float2>{pu[0], pu[1], pu[2]},
            V3<float2>{pd[t][0], pd[t][1], pd[t][2]}};
        float2 w[6];
        if (PXY) {
          w[0] = w[1] = w[2] = w[3] = make_float2(1.f, 1.f);
        } else {
          const float wyp = (c.pery || y + 1 < ny) ? 1.f : 0.f, wym = (c.pery || y - 1 >= 0) ? 1.f : 0.f;
          w[0] = make_float2((c.perx || x + 1 < nx) ? 1.f : 0.f, (c.perx || x + 3 < nx) ? 1.f : 0.f);
          w[1] = make_float2((c.perx || x - 1 >= 0) ? 1.f : 0.f, 1.f);
          w[2] = make_float2(wyp, wyp);
          w[3] = make_float2(wym, wym);
        }
        const float wzu = above ? 1.f : 0.f, wzd = has_below ? 1.f : 0.f;
        w[4] = make_float2(wzu, wzu);
        w[5] = make_float2(wzd, wzd);
        res[t] = site_update<POT, FLIP, PXY, CHIRAL, FIELD, float2, SINGLE>(m, n, nb, w, sid, sn, c.elecE, ld, c.av,
                                                                           c.T, c.invT);
      }
#pragma unroll
      for (int t = 0; t < TPT; t++) {
        if (!live[t]) continue;
        const int y = y0 + rr[t];
        const float2 fin[3] = {make_float2(res[t].n.x.x, v1 ? res[t].n.x.y : o[t][0].y),
                               make_float2(res[t].n.y.x, v1 ? res[t].n.y.y : o[t][1].y),
                               make_float2(res[t].n.z.x, v1 ? res[t].n.z.y : o[t][2].y)};
        // in-place store of the pair (half-row of parity h of row y, plane zw), then the ghosts of edge sites
        float *row0 = a.out + R.off + ((long long)zw * R.py + (y + GY)) * R.px + h * R.hp + GH;
        if (v1) {
#pragma unroll
          for (int q = 0; q < 3; q++) *reinterpret_cast<float2 *>(row0 + q * cs + jl) = fin[q];
        } else {
#pragma unroll
          for (int q = 0; q < 3; q++) row0[q * cs + jl] = fin[q].x;
        }
        const bool gx = c.perx && (jl == 0 || jl + 1 >= (nx >> 1) - 1);
        const bool gy = c.pery && (y < 2 || y >= ny - 2);
        if (gx || gy)
          pass_ghosts(row0, cs, R.px, fin[0].x, fin[1].x, fin[2].x, fin[0].y, fin[1].y, fin[2].y, v1, jl, nx, ny, y,
                      c.perx, c.pery);
        accepted += (res[t].rot.x ? 1u : 0u) + (v1 && res[t].rot.y ? 1u : 0u);
        // the other-parity cells of the pair: the colour-0 sites measured below, and the next step's -z neighbours
        const float *pn_src = cs_k + ((rr[t] + 1) * 2 + (h ^ 1)) * HALF + jb;
        float2 pn[3];
#pragma unroll
        for (int q = 0; q < 3; q++) pn[q] = *reinterpret_cast<const float2 *>(pn_src + q * PF);
        if (measure) {
          const float2 eb = __ffma2_rn(make_float2(2.f, 2.f), res[t].bond, res[t].single);
          float e = v1 ? eb.x + eb.y : eb.x;
          // the colour-0 sites in the same cells of the other half-row (pn): x0 + 4 p + (h ^ 1) + 2 e
          float2 va[3], vb[3];
#pragma unroll
          for (int q = 0; q < 3; q++) {
            va[q] = pn[q];
            vb[q] = fin[q];
          }
          const int xa0 = x0 + 4 * p + (h ^ 1);
          const bool a0 = xa0 < nx, a1 = xa0 + 2 < nx;
          if (SINGLE) {
            const float2 sa = single_energy<FIELD>(m, V3<float2>{va[0], va[1], va[2]}, sid, sn, c.elecE);
            if (a0) e += sa.x;
            if (a1) e += sa.y;
          }
          if (!(v1 && a0 && a1)) {  // ragged right edge: lanes outside the lattice count nothing
#pragma unroll
            for (int q = 0; q < 3; q++) {
              vb[q].y = v1 ? vb[q].y : 0.f;
              va[q].x = a0 ? va[q].x : 0.f;
              va[q].y = a1 ? va[q].y : 0.f;
            }
          }
          n_meas += 1 + (int)v1 + (int)a0 + (int)a1;
          float2 mo[9];
          pair_moments(mo, vb, va);
          dacc[0] += (double)e;
#pragma unroll
          for (int q = 0; q < 9; q++) dacc[q + 1] += (double)(mo[q].x + mo[q].y);
        }
#pragma unroll
        for (int q = 0; q < 3; q++) pd[t][q] = pn[q];
      }
    };
    if (single_terms)
      step(std::true_type{});
    else
      step(std::false_type{});
  }

  if (!ok) {
    if (tid == 0) {
      atomicOr(a.err, 1u);
      for (int q = max(waited + 1, last_issued - NSLP + 1); q <= last_issued; q++) {
        if (!plane_exists(q) || (a.skip_first_load && q == pbeg)) continue;
        const int lp = q - pbeg;
        mbar_wait_bounded(&bars[(unsigned)lp % NSLP], ((unsigned)lp / NSLP) & 1u, a.timeout_ns);
      }
    }
    __syncthreads();
    return;
  }

  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&a.st[it.rep].acc, (unsigned long long)wsum);
  if (measure) {
    // raw moments -> sum of q = 1.5 v_a v_b - 0.5 delta_ab (partials 1..6: xx, xy, xz, yy, yz, zz)
#pragma unroll
    for (int q = 1; q <= 6; q++) dacc[q] *= 1.5;
    dacc[1] -= 0.5 * n_meas;
    dacc[4] -= 0.5 * n_meas;
    dacc[6] -= 0.5 * n_meas;
    __shared__ double red[NT / 32][kPartials];
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < kPartials; q++) {
      double v = dacc[q];
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

template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD, int TY, int NT, int MINB, int TPT,
          int TX = 64>
cudaError_t launch_pass_one(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  auto k = k_sweep_pass<POT, GEO, FLIP, PXY, CHIRAL, FIELD, TY, NT, MINB, TPT, TX>;
  if (l.prepare) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem);
  k<<<l.n_items, NT, l.smem, l.stream>>>(m, a);
  return cudaGetLastError();
}

// Pass tile configurations (cfg numbering continues the fused kernel's): 2: 64 x 16, 256 threads, 3 CTAs/SM;
// 3: 64 x 32, 512 threads, 1 CTA/SM; 4: 64 x 16, 256 threads, 2 CTAs/SM; 5: 64 x 16, 128 threads with two pair
// tasks each (rows r and r + 8), 3 CTAs/SM.
template <int POT, int GEO, bool FLIP, bool PXY, bool CHIRAL, bool FIELD>
cudaError_t launch_pass_cfg(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.cfg == 3) return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 32, 512, 1, 1>(m, a, l);
  if (l.cfg == 4) return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 256, 2, 1>(m, a, l);
  if (l.cfg == 5) return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 128, 3, 2>(m, a, l);
  if (l.cfg == 6) return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 128, 5, 1, 32>(m, a, l);
  return launch_pass_one<POT, GEO, FLIP, PXY, CHIRAL, FIELD, 16, 256, 3, 1>(m, a, l);
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
