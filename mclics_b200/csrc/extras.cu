// Extra order parameters of one replica on the device (src/parameter_order.cpp:129-245): polarisation P,
// splay-vector magnitude <dtheta>, mean divergence <div n>, and the radial orders Sr, Pr about the lattice centre
// (sphere) and the z axis through it (cylinder). One thread per site reads the site and its six neighbours with the
// sweep's presence rules (free axes and empty sites), forms the per-site terms in FP32 with the reference's
// operations, and block partials are summed in FP64; a second kernel reduces the blocks in a fixed order.
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "eigen3.cuh"
#include "engine.h"
#include "launch.h"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {

// Partial sums per block: splay vector (3), bonds, sum of div, sites with a divergence, sum of d.n, valid sites,
// Sr / Pr / count about the centre, Sr / Pr / count about the axis.
constexpr int kExtra = 14;

template <int GEO>
__global__ void __launch_bounds__(kThreads) k_extras(RepDesc R, const float *__restrict__ dir,
                                                     const uint8_t *__restrict__ pt, const float *__restrict__ nrm,
                                                     float d0, float d1, float d2, double *__restrict__ partials) {
  double acc[kExtra];
#pragma unroll
  for (int k = 0; k < kExtra; k++) acc[k] = 0.0;
  const long long N = (long long)R.nx * R.ny * R.nz;
  const long long q = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (q < N) {
    const unsigned qq = (unsigned)q, row = qq / (unsigned)R.nx;
    const int x = (int)(qq - row * (unsigned)R.nx);
    const int z = (int)(row / (unsigned)R.ny), y = (int)(row - (unsigned)z * (unsigned)R.ny);
    Vec3 a, nb[6], s;
    float w[6];
    int sid;
    if (gather_site_rows<GEO>(R, dir, pt, nrm, x, y, z, a, nb, w, sid, s)) {
      // splay vector (parameter_order.cpp:158-170): every present bond, r the bond direction
#pragma unroll
      for (int d = 0; d < 6; d++) {
        if (w[d] == 0.f) continue;
        const Vec3 &b = nb[d];
        const int ax = d >> 1;
        const float sg = (d & 1) ? -1.f : 1.f;
        // a.r and b.r for r = sg e_ax: the reference's sums with components 0 and +-1 are these exactly
        const float ra = sg * (ax == 0 ? a.x : (ax == 1 ? a.y : a.z));
        const float rb = sg * (ax == 0 ? b.x : (ax == 1 ? b.y : b.z));
        const float ab = a.x * b.x + a.y * b.y + a.z * b.z;
        acc[0] += 0.5 * (double)(b.x * rb - a.x * ra + a.x * ab * rb - b.x * ab * ra);
        acc[1] += 0.5 * (double)(b.y * rb - a.y * ra + a.y * ab * rb - b.y * ab * ra);
        acc[2] += 0.5 * (double)(b.z * rb - a.z * ra + a.z * ab * rb - b.z * ab * ra);
        acc[3] += 1.0;
      }
      // divergence (parameter_order.cpp:192-210): per axis central or one-sided difference
      double div = 0.0;
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        double dd = 0.0;
        int cnt = 0;
#pragma unroll
        for (int sgi = 0; sgi < 2; sgi++) {  // bond 2 ax is +1, 2 ax + 1 is -1
          const int d = 2 * ax + (sgi == 0 ? 1 : 0);
          if (w[d] == 0.f) continue;
          const float sg = sgi == 0 ? -1.f : 1.f;
          const float bc = ax == 0 ? nb[d].x : (ax == 1 ? nb[d].y : nb[d].z);
          const float ac = ax == 0 ? a.x : (ax == 1 ? a.y : a.z);
          dd += (double)(sg * (bc - ac));
          cnt++;
        }
        if (cnt) div += dd / cnt;
      }
      acc[4] = div;
      acc[5] = 1.0;
      // polarisation (parameter_order.cpp:135-139)
      acc[6] = (double)(d0 * a.x + d1 * a.y + d2 * a.z);
      acc[7] = 1.0;
      // radial orders (parameter_order.cpp:225-240)
      const float cx = (float)(R.nx / 2), cy = (float)(R.ny / 2), cz = (float)(R.nz / 2);
#pragma unroll
      for (int cyl = 0; cyl < 2; cyl++) {
        const float rx = x - cx, ry = y - cy, rz = cyl ? 0.f : z - cz;
        const float r = sqrtf(rx * rx + ry * ry + rz * rz);
        if (r < 0.5f) continue;
        const double c = (a.x * rx + a.y * ry + a.z * rz) / r;
        acc[8 + 3 * cyl] = 1.5 * c * c - 0.5;
        acc[9 + 3 * cyl] = c;
        acc[10 + 3 * cyl] = 1.0;
      }
    }
  }
  __shared__ double red[kThreads / 32][kExtra];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kExtra; k++) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kExtra) {
    double v = 0.0;
    for (int w2 = 0; w2 < kThreads / 32; w2++) v += red[w2][threadIdx.x];
    partials[(long long)blockIdx.x * kExtra + threadIdx.x] = v;
  }
}

__global__ void k_extras_reduce(const double *__restrict__ partials, int n_blocks, double *__restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kExtra) return;
  double v = 0.0;
  for (int b = 0; b < n_blocks; b++) v += partials[(long long)b * kExtra + k];
  out[k] = v;
}

// Local order parameter of every site (src/parameter_order.cpp:75-127): Q over the site and its present
// neighbours, accumulated in FP32 in the reference's visiting order (-x, -y, -z, the site, +z, +y, +x), divided by
// 2 x points, then the largest eigenvalue (FP64 Jacobi). NaN on empty sites. out: nx ny nz floats, reference order.
template <int GEO>
__global__ void __launch_bounds__(kThreads) k_local_order(RepDesc R, const float *__restrict__ dir,
                                                          const uint8_t *__restrict__ pt,
                                                          const float *__restrict__ nrm, float *__restrict__ out) {
  const long long N = (long long)R.nx * R.ny * R.nz;
  const long long q = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (q >= N) return;
  const unsigned qq = (unsigned)q, row = qq / (unsigned)R.nx;
  const int x = (int)(qq - row * (unsigned)R.nx);
  const int z = (int)(row / (unsigned)R.ny), y = (int)(row - (unsigned)z * (unsigned)R.ny);
  Vec3 a, nb[6], s;
  float w[6];
  int sid;
  if (!gather_site_rows<GEO>(R, dir, pt, nrm, x, y, z, a, nb, w, sid, s)) {
    out[q] = __int_as_float(0x7fc00000);
    return;
  }
  float Q[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int points = 0;
  const int order[7] = {1, 3, 5, -1, 4, 2, 0};  // -1: the site itself
#pragma unroll
  for (int o = 0; o < 7; o++) {
    const int d = order[o];
    if (d >= 0 && w[d] == 0.f) continue;
    const Vec3 v = d < 0 ? a : nb[d];
    const float c[3] = {v.x, v.y, v.z};
#pragma unroll
    for (int l = 0; l < 3; l++) {
#pragma unroll
      for (int m = 0; m <= l; m++) Q[3 * m + l] = (float)((double)Q[3 * m + l] + 3.0 * (double)__fmul_rn(c[l], c[m]));
      Q[4 * l] = __fadd_rn(Q[4 * l], -1.f);
    }
    points++;
  }
  const double den = 2.0 * points;
  double qd[6] = {(float)(Q[0] / den), (float)(Q[1] / den), (float)(Q[2] / den),
                  (float)(Q[4] / den), (float)(Q[5] / den), (float)(Q[8] / den)};
  double v3[3];
  out[q] = (float)largest_eigen3(qd, v3);
}

}  // namespace mcl

using namespace mcl;

#define CKX(call)                                        \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

extern "C" int mcl_measure_extras(mcl_engine *e, int replica, const double director[3], mcl_extras *out) {
  if (!e || !director || !out) return fail(MCL_ERR_ARG, "mcl_measure_extras: null argument");
  if (replica < 0 || replica >= e->n_rep) return fail(MCL_ERR_ARG, "replica %d outside 0..%d", replica, e->n_rep - 1);
  if (!e->geometry_set) return fail(MCL_ERR_STATE, "custom geometry: call mcl_set_geometry first");
  const RepDesc &D = e->desc[replica];
  const long long N = (long long)D.nx * D.ny * D.nz;
  const int n_blocks = (int)((N + kThreads - 1) / kThreads);
  if (!e->d_xpart) {  // first call: scratch for the largest replica
    const long long most = (e->max_sites + kThreads - 1) / kThreads;
    CKX(cudaMalloc(&e->d_xpart, (size_t)(most * kExtra + kExtra) * sizeof(double)));
  }
  double *partials = e->d_xpart, *sums = e->d_xpart + (size_t)n_blocks * kExtra;
  const LaunchCtx c = e->ctx();
  const float d0 = (float)director[0], d1 = (float)director[1], d2 = (float)director[2];
  switch (e->geo) {
    case GEO_BULK:
      k_extras<GEO_BULK><<<n_blocks, kThreads, 0, c.stream>>>(D, c.dir, c.pt, c.nrm, d0, d1, d2, partials);
      break;
    case GEO_SLAB:
      k_extras<GEO_SLAB><<<n_blocks, kThreads, 0, c.stream>>>(D, c.dir, c.pt, c.nrm, d0, d1, d2, partials);
      break;
    default:
      k_extras<GEO_PT><<<n_blocks, kThreads, 0, c.stream>>>(D, c.dir, c.pt, c.nrm, d0, d1, d2, partials);
  }
  CKX(cudaGetLastError());
  k_extras_reduce<<<1, 32, 0, c.stream>>>(partials, n_blocks, sums);
  CKX(cudaGetLastError());
  e->launches += 2;
  double v[kExtra];
  CKX(cudaMemcpyAsync(v, sums, sizeof v, cudaMemcpyDeviceToHost, c.stream));
  CKX(cudaStreamSynchronize(c.stream));
  out->P = v[7] > 0 ? std::fabs(v[6]) / v[7] : 0.0;
  out->dtheta = v[3] > 0 ? 1.5 * std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / v[3] : 0.0;
  out->divn = v[5] > 0 ? v[4] / v[5] : 0.0;
  out->Sr_sph = v[10] > 0 ? v[8] / v[10] : 0.0;
  out->Pr_sph = v[10] > 0 ? v[9] / v[10] : 0.0;
  out->Sr_cyl = v[13] > 0 ? v[11] / v[13] : 0.0;
  out->Pr_cyl = v[13] > 0 ? v[12] / v[13] : 0.0;
  return MCL_OK;
}

extern "C" int mcl_local_order(mcl_engine *e, int replica, float *S) {
  if (!e || !S) return fail(MCL_ERR_ARG, "mcl_local_order: null argument");
  if (replica < 0 || replica >= e->n_rep) return fail(MCL_ERR_ARG, "replica %d outside 0..%d", replica, e->n_rep - 1);
  if (!e->geometry_set) return fail(MCL_ERR_STATE, "custom geometry: call mcl_set_geometry first");
  const RepDesc &D = e->desc[replica];
  const long long N = (long long)D.nx * D.ny * D.nz;
  const int n_blocks = (int)((N + kThreads - 1) / kThreads);
  const LaunchCtx c = e->ctx();
  float *out = e->d_stage;  // max_sites x 3 floats, free between uploads and downloads
  switch (e->geo) {
    case GEO_BULK:
      k_local_order<GEO_BULK><<<n_blocks, kThreads, 0, c.stream>>>(D, c.dir, c.pt, c.nrm, out);
      break;
    case GEO_SLAB:
      k_local_order<GEO_SLAB><<<n_blocks, kThreads, 0, c.stream>>>(D, c.dir, c.pt, c.nrm, out);
      break;
    default:
      k_local_order<GEO_PT><<<n_blocks, kThreads, 0, c.stream>>>(D, c.dir, c.pt, c.nrm, out);
  }
  CKX(cudaGetLastError());
  e->launches++;
  CKX(cudaMemcpyAsync(S, out, (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  CKX(cudaStreamSynchronize(c.stream));
  return MCL_OK;
}
