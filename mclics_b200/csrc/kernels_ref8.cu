// Reference-order sweep for decision-by-decision replay: the reference CPU's 8 sublattices (parities
// (i%2, j%2, k%2), visited with i fastest: src/evolve.cpp:106-119), one launch per sublattice, and the reference
// CPU's float/double arithmetic (physics_exact.cuh). This file is compiled with -fmad=false.
#include <cuda_runtime.h>
#include <math.h>

#include "common.cuh"
#include "launch.h"
#include "physics_exact.cuh"
#include "site_access.cuh"

namespace mcl {

template <int POT, int GEO>
__global__ void __launch_bounds__(kThreads) k_sweep_ref8(ModelDev m, const RepDesc *__restrict__ reps,
                                                         RepState *__restrict__ st, float *__restrict__ dir,
                                                         const uint8_t *__restrict__ pt, const float *__restrict__ nrm,
                                                         const unsigned long long *__restrict__ sweep_ctr, int tick,
                                                         const int *__restrict__ blk_rep,
                                                         const long long *__restrict__ blk_base,
                                                         uint8_t *__restrict__ dec) {
  const int rep = blk_rep[blockIdx.x];
  const RepDesc R = reps[rep];
  const long long q = blk_base[blockIdx.x] + threadIdx.x;
  const int bx = (R.nx + 1) / 2, by = (R.ny + 1) / 2, bz = (R.nz + 1) / 2;
  const int di = tick % 2, dj = (tick / 2) % 2, dk = tick / 4;
  unsigned accepted = 0;
  if (q < (long long)bx * by * bz) {
    const int x = di + 2 * (int)(q % bx), y = dj + 2 * (int)((q / bx) % by), z = dk + 2 * (int)(q / ((long long)bx * by));
    Vec3 n3, nb3[6], s3;
    unsigned present;
    int sid;
    if (x < R.nx && y < R.ny && z < R.nz && gather_site<GEO>(R, dir, pt, nrm, x, y, z, n3, nb3, present, sid, s3)) {
      const float n[3] = {n3.x, n3.y, n3.z};
      float nb[6][3];
      for (int d = 0; d < 6; d++) {
        nb[d][0] = nb3[d].x;
        nb[d][1] = nb3[d].y;
        nb[d][2] = nb3[d].z;
      }
      const float s[3] = {s3.x, s3.y, s3.z};
      const RepState S = st[rep];
      const float T = S.T;
      const long long site = site_linear(R, x, y, z);
      const bool fl = m.flip;
      const Draw r = site_draw(R.seed, *sweep_ctr, x, y, z, R.nx, R.ny, fl);
      // src/evolve.cpp:153-176 with the reference's double intermediate values
      const double u1 = unif_d(r.f1, fl);
      const float va = (float)((2 * u1 - 1) * (double)S.ang_var);
      const float ang = (float)(M_PI * (double)va);
      const float c = cosf(ang), sn = sinf(ang);
      float nn[3];
      const int axis = rotation_axis(r.f2, fl);
      if (axis == 0) {
        nn[0] = n[0];
        nn[1] = n[1] * c + n[2] * sn;
        nn[2] = n[2] * c - n[1] * sn;
      } else if (axis == 1) {
        nn[0] = n[0] * c - n[2] * sn;
        nn[1] = n[1];
        nn[2] = n[2] * c + n[0] * sn;
      } else {
        nn[0] = n[0] * c + n[1] * sn;
        nn[1] = n[1] * c - n[0] * sn;
        nn[2] = n[2];
      }
      const float norm = sqrtf(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
      nn[0] /= norm;
      nn[1] /= norm;
      nn[2] /= norm;
      const float e_old = exact::site_energy<POT>(m, n, nb, present, sid, s, S.elecE);
      const float e_new = exact::site_energy<POT>(m, nn, nb, present, sid, s, S.elecE);
      float cur[3] = {n[0], n[1], n[2]};
      float e_cur = e_old;
      uint8_t d = 0x80;
      const float u3 = unif(r.f3, fl);
      if (T > 0 ? u3 < expf(-(e_new - e_old) / T) : e_new <= e_old) {
        cur[0] = nn[0];
        cur[1] = nn[1];
        cur[2] = nn[2];
        e_cur = e_new;
        accepted = 1;
        d |= 1;
      }
      if (m.flip) {
        const float f[3] = {-cur[0], -cur[1], -cur[2]};
        const float e_flip = exact::site_energy<POT>(m, f, nb, present, sid, s, S.elecE);
        const float u4 = unif(r.f4, fl);
        if (T > 0 ? u4 < expf(-(e_flip - e_cur) / T) : e_flip <= e_cur) {
          cur[0] = f[0];
          cur[1] = f[1];
          cur[2] = f[2];
          d |= 2;
        }
      }
      if (d & 3) {
        dir[dir_index(R, 0, x, y, z)] = cur[0];
        dir[dir_index(R, 1, x, y, z)] = cur[1];
        dir[dir_index(R, 2, x, y, z)] = cur[2];
      }
      if (dec) dec[R.site_off + site] = d;
    }
  }
  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(&st[rep].acc, (unsigned long long)wsum);
}

template <int POT>
static void ref8_pot(const LaunchCtx &c, int geo, const BlockTable &t, int tick) {
  dim3 g(t.n_blocks), b(kThreads);
  switch (geo) {
    case GEO_BULK:
      k_sweep_ref8<POT, GEO_BULK><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr,
                                                         tick, t.rep, t.base, c.decisions);
      break;
    case GEO_SLAB:
      k_sweep_ref8<POT, GEO_SLAB><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr,
                                                         tick, t.rep, t.base, c.decisions);
      break;
    default:
      k_sweep_ref8<POT, GEO_PT><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr,
                                                       tick, t.rep, t.base, c.decisions);
  }
}

cudaError_t launch_sweep_ref8(const LaunchCtx &c, int geo, const BlockTable &boxes) {
  if (boxes.n_blocks == 0) return cudaSuccess;
  for (int tick = 0; tick < 8; tick++) {
    if (c.model.potential == POT_GHRL)
      ref8_pot<POT_GHRL>(c, geo, boxes, tick);
    else if (c.model.potential == POT_PEAR)
      ref8_pot<POT_PEAR>(c, geo, boxes, tick);
    else
      ref8_pot<POT_LL>(c, geo, boxes, tick);
  }
  return cudaGetLastError();
}

}  // namespace mcl
