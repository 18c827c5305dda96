// Simple (untiled) device kernels: two-colour sweep, observables, per-sweep finalisation, ghost cells and the
// AoS <-> padded-SoA conversion used at the host boundary.
#include <cuda_runtime.h>

#include "common.cuh"
#include "eigen3.cuh"
#include "launch.h"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {

// ------------------------------------------------------------------------------------------------------------
// Two-colour sweep, one thread per site of colour `colour` (parity of x + y + z). Same trial move as the
// reference (src/evolve.cpp:133-207), draws from Philox(seed, sweep, site).
template <int POT, int GEO>
__global__ void __launch_bounds__(kThreads) k_sweep_color(ModelDev m, const RepDesc *__restrict__ reps,
                                                          RepState *__restrict__ st, float *__restrict__ dir,
                                                          const uint8_t *__restrict__ pt,
                                                          const float *__restrict__ nrm,
                                                          const unsigned long long *__restrict__ sweep_ctr, int colour,
                                                          const int *__restrict__ blk_rep,
                                                          const long long *__restrict__ blk_base,
                                                          uint8_t *__restrict__ dec) {
  const int rep = blk_rep[blockIdx.x];
  const RepDesc R = reps[rep];
  const long long q = blk_base[blockIdx.x] + threadIdx.x;
  const int hx = (R.nx + 1) >> 1;
  unsigned accepted = 0;
  const long long total = (long long)hx * R.ny * R.nz;
  if (q < total) {
    const int xh = (int)(q % hx);
    const long long row = q / hx;
    const int y = (int)(row % R.ny), z = (int)(row / R.ny);
    const int x = 2 * xh + ((colour + y + z) & 1);
    Vec3 n, nb[6], s;
    float w[6];
    int sid;
    if (x < R.nx && gather_site_w<GEO>(R, dir, pt, nrm, x, y, z, n, nb, w, sid, s)) {
      const RepState S = st[rep];
      const float T = S.T, invT = 1.f / T;
      const long long site = site_linear(R, x, y, z);
      const Draw d = site_draw(R.seed, *sweep_ctr, x, y, z, R.nx, R.ny, m.flip);
      const LaneDraw<float> ld = lane_draw(d, m.flip);
      const SiteResultT<float> r =
          m.flip ? site_update<POT, true, false, true, true, float>(m, n, nb, w, sid, s, S.elecE, ld, S.ang_var, T, invT)
                 : site_update<POT, false, false, true, true, float>(m, n, nb, w, sid, s, S.elecE, ld, S.ang_var, T, invT);
      accepted = r.rot ? 1u : 0u;
      if (r.rot || r.flip) {
        dir[dir_index(R, 0, x, y, z)] = r.n.x;
        dir[dir_index(R, 1, x, y, z)] = r.n.y;
        dir[dir_index(R, 2, x, y, z)] = r.n.z;
      }
      if (dec) dec[R.site_off + site] = (uint8_t)(0x80u | (r.rot ? 1u : 0u) | (r.flip ? 2u : 0u));
    }
  }
  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(&st[rep].acc, (unsigned long long)wsum);
}

// ------------------------------------------------------------------------------------------------------------
// Observables of the current state: per block sums of the site energies, (3 n n - I)/2 and n, in FP64.
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int POT, int GEO>
__global__ void __launch_bounds__(kThreads) k_observe(ModelDev m, const RepDesc *__restrict__ reps,
                                                      const RepState *__restrict__ st, const float *__restrict__ dir,
                                                      const uint8_t *__restrict__ pt, const float *__restrict__ nrm,
                                                      const int *__restrict__ blk_rep,
                                                      const long long *__restrict__ blk_base,
                                                      double *__restrict__ partials) {
  const int rep = blk_rep[blockIdx.x];
  const RepDesc R = reps[rep];
  const long long q = blk_base[blockIdx.x] + threadIdx.x;
  double acc[kPartials];
#pragma unroll
  for (int k = 0; k < kPartials; k++) acc[k] = 0.0;
  if (q < (long long)R.nx * R.ny * R.nz) {
    const int x = (int)(q % R.nx);
    const long long row = q / R.nx;
    const int y = (int)(row % R.ny), z = (int)(row / R.ny);
    Vec3 n, nb[6], s;
    float w[6];
    int sid;
    if (gather_site_w<GEO>(R, dir, pt, nrm, x, y, z, n, nb, w, sid, s)) {
      acc[0] = (double)site_energy<POT>(m, n, nb, w, sid, s, st[rep].elecE);
      const double nx = n.x, ny = n.y, nz = n.z;
      acc[1] = 1.5 * nx * nx - 0.5;
      acc[2] = 1.5 * nx * ny;
      acc[3] = 1.5 * nx * nz;
      acc[4] = 1.5 * ny * ny - 0.5;
      acc[5] = 1.5 * ny * nz;
      acc[6] = 1.5 * nz * nz - 0.5;
      acc[7] = nx;
      acc[8] = ny;
      acc[9] = nz;
    }
  }
  __shared__ double red[kThreads / 32][kPartials];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kPartials; k++) {
    double v = warp_sum_d(acc[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kPartials) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; w++) v += red[w][threadIdx.x];
    partials[(long long)blockIdx.x * kPartials + threadIdx.x] = v;
  }
}

// ------------------------------------------------------------------------------------------------------------
// One block per replica: deterministic reduction of the replica's partials, S and director by Jacobi, ang_var
// adaptation (src/evolve.cpp:211-220; skipped when adapt = 0), optional series record, reset of the acceptance
// counter. The last
// block to finish advances the global sweep counter and the series length. measure: 0 none, 1 append to the
// series, 2 probe (record the current state into series[rep]; no adaptation, counters untouched). gsums (z-slab
// processes): the observables and accepted rotations already summed over all processes (kZslabSums per replica)
// replace the local partials and the local acceptance counter.
__global__ void __launch_bounds__(kThreads) k_finalize(const RepDesc *__restrict__ reps, RepState *__restrict__ st,
                                                       const int *__restrict__ obs_first,
                                                       const double *__restrict__ partials, int measure,
                                                       ObsRecord *__restrict__ series, int *__restrict__ series_len,
                                                       unsigned long long *__restrict__ sweep_ctr,
                                                       unsigned int *__restrict__ done_ctr, int n_replicas,
                                                       int adapt, const double *__restrict__ gsums) {
  const int rep = blockIdx.x;
  __shared__ double red[kThreads / 32][kPartials];
  __shared__ double tot[kPartials];
  const unsigned long long sweep = *sweep_ctr;
  const int slen = *series_len;
  if (measure && gsums) {
    if (threadIdx.x < kPartials) tot[threadIdx.x] = gsums[(long long)rep * kZslabSums + threadIdx.x];
    __syncthreads();
  } else if (measure) {
    double acc[kPartials];
#pragma unroll
    for (int k = 0; k < kPartials; k++) acc[k] = 0.0;
    for (int b = obs_first[rep] + threadIdx.x; b < obs_first[rep + 1]; b += kThreads)
#pragma unroll
      for (int k = 0; k < kPartials; k++) acc[k] += partials[(long long)b * kPartials + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kPartials; k++) {
      double v = warp_sum_d(acc[k]);
      if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kPartials) {
      double v = 0.0;
      for (int w = 0; w < kThreads / 32; w++) v += red[w][threadIdx.x];
      tot[threadIdx.x] = v;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const RepDesc R = reps[rep];
    const RepState S = st[rep];
    const double nv = R.n_valid;
    const bool probe = measure == 2;  // measurement of the current state only: no adaptation, no counters
    double a = S.pad;
    float av = S.ang_var;
    const double nacc = gsums ? gsums[(long long)rep * kZslabSums + kPartials] : (double)S.acc;
    if (!probe) {
      a = nacc / nv;
      if (!adapt) {
      } else if (1.0 * nacc / nv < 0.5) {
        av = (float)((double)av * 0.99);
        if (av < 0.01) av = 0.01f;
      } else if (1.0 * nacc / nv > 0.5) {
        av = (float)((double)av / 0.99);
        if (av > 1.0) av -= 0.5f;
      }
      st[rep].ang_var = av;
      st[rep].pad = (float)a;
      st[rep].acc = 0ull;
    }
    if (measure) {
      ObsRecord o;
      o.energy = tot[0] / nv;
      for (int k = 0; k < 6; k++) o.q[k] = tot[1 + k] / nv;
      double vec[3];
      o.S = largest_eigen3(o.q, vec);
      for (int k = 0; k < 3; k++) {
        o.director[k] = vec[k];
        o.nsum[k] = tot[7 + k];
      }
      o.n_valid = nv;
      o.acceptance = a;
      o.ang_var = av;
      o.sweep = (double)sweep;
      series[(long long)slen * n_replicas + rep] = o;
    }
    if (!probe) {
      __threadfence();
      const unsigned prev = atomicAdd(done_ctr, 1u);
      if (prev == (unsigned)gridDim.x - 1) {
        *done_ctr = 0u;
        *sweep_ctr = sweep + 1ull;
        if (measure) *series_len = slen + 1;
        __threadfence();
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------------------
// Ghost cells of periodic axes. Pass 0 fills the x ghosts of every row; pass 1 the y ghost rows (including
// their x ghosts, so corners are consistent).
__global__ void k_ghosts_x(const RepDesc *__restrict__ reps, int n_rep, float *__restrict__ dir) {
  const int rep = blockIdx.y;
  if (rep >= n_rep) return;
  const RepDesc R = reps[rep];
  if (!R.periodic[0]) return;
  const long long rows = 3ll * R.nz * R.ny;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < rows * 4; q += (long long)gridDim.x * blockDim.x) {
    const long long row = q >> 2;
    const int g = (int)(q & 3);
    const int c = (int)(row / ((long long)R.nz * R.ny));
    const long long zr = row % ((long long)R.nz * R.ny);
    const int z = (int)(zr / R.ny), y = (int)(zr % R.ny);
    const int gx = g < 2 ? g - 2 : R.nx + g - 2;      // -2, -1, nx, nx+1
    const int sx = g < 2 ? R.nx + g - 2 : g - 2;      // nx-2, nx-1, 0, 1
    if (sx < 0 || sx >= R.nx) continue;
    dir[dir_index(R, c, gx, y, z)] = dir[dir_index(R, c, sx, y, z)];
  }
}

__global__ void k_ghosts_y(const RepDesc *__restrict__ reps, int n_rep, float *__restrict__ dir) {
  const int rep = blockIdx.y;
  if (rep >= n_rep) return;
  const RepDesc R = reps[rep];
  if (!R.periodic[1]) return;
  const int w = R.nx + 4;  // x from -2 to nx+1
  const long long cols = 3ll * R.nz * w;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < cols * 4; q += (long long)gridDim.x * blockDim.x) {
    const long long col = q >> 2;
    const int g = (int)(q & 3);
    const int c = (int)(col / ((long long)R.nz * w));
    const long long zr = col % ((long long)R.nz * w);
    const int z = (int)(zr / w), x = (int)(zr % w) - 2;
    const int gy = g < 2 ? g - 2 : R.ny + g - 2;
    const int sy = g < 2 ? R.ny + g - 2 : g - 2;
    if (sy < 0 || sy >= R.ny) continue;
    dir[dir_index(R, c, x, gy, z)] = dir[dir_index(R, c, x, sy, z)];
  }
}

// AoS (3 floats per site, x fastest) <-> padded SoA of one replica.
__global__ void k_unpack(RepDesc R, const float *__restrict__ aos, float *__restrict__ dir) {
  const long long N = (long long)R.nx * R.ny * R.nz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(q % R.nx);
    const long long row = q / R.nx;
    const int y = (int)(row % R.ny), z = (int)(row / R.ny);
    for (int c = 0; c < 3; c++) dir[dir_index(R, c, x, y, z)] = aos[3 * q + c];
  }
}

// Random initial condition of one replica (random_director per site; empty sites of a point-type geometry (0, 0, 1)).
__global__ void k_random_ic(RepDesc R, const uint8_t *__restrict__ pt, unsigned long long seed, float *__restrict__ dir) {
  const long long N = (long long)R.nx * R.ny * R.nz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(q % R.nx);
    const long long row = q / R.nx;
    const int y = (int)(row % R.ny), z = (int)(row / R.ny);
    float n[3] = {0.f, 0.f, 1.f};
    if (!pt || pt[R.site_off + q] != 0) random_director(seed, (uint32_t)q, n);
    for (int c = 0; c < 3; c++) dir[dir_index(R, c, x, y, z)] = n[c];
  }
}

__global__ void k_pack(RepDesc R, const float *__restrict__ dir, float *__restrict__ aos) {
  const long long N = (long long)R.nx * R.ny * R.nz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(q % R.nx);
    const long long row = q / R.nx;
    const int y = (int)(row % R.ny), z = (int)(row / R.ny);
    for (int c = 0; c < 3; c++) aos[3 * q + c] = dir[dir_index(R, c, x, y, z)];
  }
}

// ------------------------------------------------------------------------------------------------------------
template <int POT>
static void sweep_color_pot(const LaunchCtx &c, int geo, const BlockTable &t, int colour) {
  dim3 g(t.n_blocks), b(kThreads);
  switch (geo) {
    case GEO_BULK:
      k_sweep_color<POT, GEO_BULK><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr,
                                                          colour, t.rep, t.base, c.decisions);
      break;
    case GEO_SLAB:
      k_sweep_color<POT, GEO_SLAB><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr,
                                                          colour, t.rep, t.base, c.decisions);
      break;
    default:
      k_sweep_color<POT, GEO_PT><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr,
                                                        colour, t.rep, t.base, c.decisions);
  }
}

cudaError_t launch_sweep_checker2_simple(const LaunchCtx &c, int geo, const BlockTable &half) {
  if (half.n_blocks == 0) return cudaSuccess;
  for (int colour = 0; colour < 2; colour++) {
    if (c.model.potential == POT_GHRL)
      sweep_color_pot<POT_GHRL>(c, geo, half, colour);
    else if (c.model.potential == POT_PEAR)
      sweep_color_pot<POT_PEAR>(c, geo, half, colour);
    else
      sweep_color_pot<POT_LL>(c, geo, half, colour);
  }
  return cudaGetLastError();
}

template <int POT>
static void observe_pot(const LaunchCtx &c, int geo, const BlockTable &t, double *partials) {
  dim3 g(t.n_blocks), b(kThreads);
  switch (geo) {
    case GEO_BULK:
      k_observe<POT, GEO_BULK><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, t.rep, t.base, partials);
      break;
    case GEO_SLAB:
      k_observe<POT, GEO_SLAB><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, t.rep, t.base, partials);
      break;
    default:
      k_observe<POT, GEO_PT><<<g, b, 0, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, t.rep, t.base, partials);
  }
}

cudaError_t launch_observe(const LaunchCtx &c, int geo, const BlockTable &sites, double *partials) {
  if (sites.n_blocks == 0) return cudaSuccess;
  if (c.model.potential == POT_GHRL)
    observe_pot<POT_GHRL>(c, geo, sites, partials);
  else if (c.model.potential == POT_PEAR)
    observe_pot<POT_PEAR>(c, geo, sites, partials);
  else
    observe_pot<POT_LL>(c, geo, sites, partials);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const LaunchCtx &c, const BlockTable &sites, const double *partials, int measure,
                            ObsRecord *series, int *series_len, unsigned int *done_ctr, const double *gsums) {
  k_finalize<<<c.n_replicas, kThreads, 0, c.stream>>>(c.reps, c.state, sites.first, partials, measure, series,
                                                       series_len, c.sweep_ctr, done_ctr, c.n_replicas, c.adapt,
                                                       gsums);
  return cudaGetLastError();
}

// One block per replica: the replica's partials summed over its blocks (the order k_finalize uses; zeros when
// measure = 0) and its accepted rotations, kZslabSums doubles per replica.
__global__ void __launch_bounds__(kThreads) k_item_sums(const RepState *__restrict__ st,
                                                        const int *__restrict__ obs_first,
                                                        const double *__restrict__ partials, int measure,
                                                        double *__restrict__ out) {
  const int rep = blockIdx.x;
  __shared__ double red[kThreads / 32][kPartials];
  double acc[kPartials];
#pragma unroll
  for (int k = 0; k < kPartials; k++) acc[k] = 0.0;
  if (measure)
    for (int b = obs_first[rep] + threadIdx.x; b < obs_first[rep + 1]; b += kThreads)
#pragma unroll
      for (int k = 0; k < kPartials; k++) acc[k] += partials[(long long)b * kPartials + k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kPartials; k++) {
    double v = warp_sum_d(acc[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kPartials) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; w++) v += red[w][threadIdx.x];
    out[(long long)rep * kZslabSums + threadIdx.x] = v;
  }
  if (threadIdx.x == 0) out[(long long)rep * kZslabSums + kPartials] = (double)st[rep].acc;
}

cudaError_t launch_item_sums(const LaunchCtx &c, const BlockTable &items, const double *partials, int measure,
                             double *out) {
  k_item_sums<<<c.n_replicas, kThreads, 0, c.stream>>>(c.state, items.first, partials, measure, out);
  return cudaGetLastError();
}

// Boundary planes of a z-slab (replica 0) to or from the caller's plane buffers, each [component][py * px] (the
// whole padded plane, ghost cells included). pack: owned planes 1 and nz - 2 -> lo, hi; unpack: lo, hi -> halo
// planes 0 and nz - 1. A null buffer skips its side. blockIdx.y selects the side.
__global__ void k_zslab_planes(const RepDesc *__restrict__ reps, float *__restrict__ dir, float *lo, float *hi,
                               int pack) {
  const RepDesc R = reps[0];
  const long long pf = (long long)R.py * R.px;
  float *buf = blockIdx.y ? hi : lo;
  if (!buf) return;
  const int plane = pack ? (blockIdx.y ? R.nz - 2 : 1) : (blockIdx.y ? R.nz - 1 : 0);
  float *base = dir + R.off + plane * pf;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * pf;
       i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / pf, o = i - q * pf;
    if (pack)
      buf[i] = base[q * R.comp + o];
    else
      base[q * R.comp + o] = buf[i];
  }
}

cudaError_t launch_zslab_planes(const LaunchCtx &c, float *dir, float *lo, float *hi, int pack) {
  k_zslab_planes<<<dim3(148, 2), kThreads, 0, c.stream>>>(c.reps, dir, lo, hi, pack);
  return cudaGetLastError();
}

// Step input and output of mcl_sweeps_io through mapped pinned host memory (no copy-engine round trips): the
// replicas' temperatures in; the records of series rows first_row .. first_row + n_rows - 1 and the two error words
// out. The caller validates the row range against the series it has written.
__global__ void k_io_in(RepState *__restrict__ st, const float *__restrict__ host_T, int n_rep) {
  for (int r = threadIdx.x; r < n_rep; r += blockDim.x) st[r].T = host_T[r];
}

// series_len non-null (a captured graph, whose arguments are fixed): the rows are the newest n_rows, and first_row is
// ignored.
__global__ void k_io_out(const ObsRecord *__restrict__ series, long long first_row, const int *__restrict__ series_len,
                         int n_rows, int n_rep, ObsRecord *__restrict__ host_rec, const unsigned *__restrict__ err0,
                         const unsigned *__restrict__ err1, unsigned *__restrict__ host_words) {
  static_assert(sizeof(ObsRecord) % 8 == 0, "records move as 8-byte words");
  if (series_len) first_row = max(0, *series_len - n_rows);
  const long long words = (long long)n_rows * n_rep * (long long)(sizeof(ObsRecord) / 8);
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(series + first_row * n_rep);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(host_rec);
  for (long long i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  if (threadIdx.x == 0) {
    host_words[0] = err0 ? *err0 : 0u;
    host_words[1] = err1 ? *err1 : 0u;
  }
}

cudaError_t launch_io_in(cudaStream_t stream, RepState *st, const float *host_T, int n_rep) {
  k_io_in<<<1, 32, 0, stream>>>(st, host_T, n_rep);
  return cudaGetLastError();
}

cudaError_t launch_io_out(cudaStream_t stream, const ObsRecord *series, long long first_row, const int *series_len,
                          int n_rows, int n_rep, ObsRecord *host_rec, const unsigned *err0, const unsigned *err1,
                          unsigned *host_words) {
  k_io_out<<<1, kThreads, 0, stream>>>(series, first_row, series_len, n_rows, n_rep, host_rec, err0, err1,
                                       host_words);
  return cudaGetLastError();
}

cudaError_t launch_refresh_ghosts(const LaunchCtx &c, int max_ny_nz, int max_px_nz) {
  const int bx = 148;
  k_ghosts_x<<<dim3(bx, c.n_replicas), kThreads, 0, c.stream>>>(c.reps, c.n_replicas, c.dir);
  k_ghosts_y<<<dim3(bx, c.n_replicas), kThreads, 0, c.stream>>>(c.reps, c.n_replicas, c.dir);
  (void)max_ny_nz;
  (void)max_px_nz;
  return cudaGetLastError();
}

cudaError_t launch_unpack(const LaunchCtx &c, int replica, const RepDesc &R, const float *aos) {
  (void)replica;
  k_unpack<<<4 * 148, kThreads, 0, c.stream>>>(R, aos, c.dir);
  return cudaGetLastError();
}

cudaError_t launch_random_ic(const LaunchCtx &c, const RepDesc &R, unsigned long long seed) {
  k_random_ic<<<4 * 148, kThreads, 0, c.stream>>>(R, R.geo == GEO_PT ? c.pt : nullptr, seed, c.dir);
  return cudaGetLastError();
}

cudaError_t launch_pack(const LaunchCtx &c, int replica, const RepDesc &R, float *aos) {
  (void)replica;
  k_pack<<<4 * 148, kThreads, 0, c.stream>>>(R, c.dir, aos);
  return cudaGetLastError();
}

}  // namespace mcl
