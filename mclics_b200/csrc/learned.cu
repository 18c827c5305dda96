// Learned Metropolis-Hastings proposal (no counterpart in the reference).
//
// Per site the proposal reads only the neighbours: the features are the neighbour Q-tensor sum
// sum_j w_j (3 n_j n_j^T - I) / 2, divided by 6 (xx, xy, xz, yy, yz, zz), and T. A 7 -> 64 -> 64 -> 4 MLP with SiLU
// maps them to an axis mu (first three outputs, normalised) and a concentration kappa = clip(softplus(o_3),
// 1e-3, kappa_max). The proposal density is
//     q(n) = [ 0.95 kappa cosh(kappa mu.n) / sinh(kappa) + 0.05 ] / (4 pi),
// an antipodally symmetrised von Mises-Fisher density mixed with 5 % uniform; it is sampled exactly (Wood's method
// for the vMF part, a random sign, or a uniform point). Because q does not depend on the site's own director, the
// Hastings test u < exp(-dE / T) q(n_old) / q(n_new) leaves the Boltzmann distribution invariant for any weights.
//
// The MLP runs on the tensor cores: one warp evaluates 32 sites as two 16-row tiles with mma.sync m16n8k16
// (BF16 operands, FP32 accumulation); the FP32 accumulator fragments of one layer, after bias and SiLU (computed
// as h + h tanh(h), h = z / 2, in packed BF16), are used directly as the A fragments of the next layer. Weights live in shared memory, rows padded so
// that the fragment loads are free of bank conflicts.
//
// Training (maximum likelihood of the local conditional distribution, loss -log(4 pi q(n | features)) over sites
// of equilibrated plain-sweep states) runs in FP32 on the CUDA cores with the same BF16 rounding of weights,
// features and hidden activations as inference: one thread per sample for the forward and backward passes, then
// the block's weight gradients from its 64 samples in shared memory, per-block partial sums, and a fixed-order
// FP64 reduction with the Adam update.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "launch.h"
#include "sweep_fused.cuh"
#include "mlp_tc.cuh"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {

constexpr int kIn = 7, kH = 64, kOut = 4;
constexpr int kNP = kH * kIn + kH + kH * kH + kH + kOut * kH + kOut;  // 4932 parameters
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH;
static_assert(oB3 + kOut == kNP, "parameter layout");
static_assert(sizeof(mcl_mlp) == kNP * sizeof(float), "mcl_mlp must be the flat parameter vector");
constexpr float kEps = 0.05f, kKappaMin = 1e-3f;
constexpr int kFeat = 8;  // floats per sample row: 7 features, validity flag

// Weights in the layout of the tensor-core fragments: [n][k] rows (k contiguous), k padded with zeros (layer 1:
// 7 -> 16), rows padded to 24 / 72 halves (16-byte aligned rows for ldmatrix, the 8 rows of a fragment in distinct
// banks); layer 3 has 8 rows (4 used). Weights and biases of the two hidden layers are stored times 1/2 (exact in
// BF16 and FP32), so that their accumulators hold h = z / 2, the argument of the SiLU form h + h tanh(h).
struct MlpDev {
  __nv_bfloat16 w1[kH][24];
  __nv_bfloat16 w2[kH][72];
  __nv_bfloat16 w3[8][72];
  float b1[kH], b2[kH], b3[8];
};
static_assert(sizeof(MlpDev) % 16 == 0, "MlpDev is copied in 16-byte words");

// ---- host: FP32 parameters -> device layout ------------------------------------------------------------------
static uint16_t bf16_bits(float f) {  // round to nearest, ties to even
  uint32_t u;
  memcpy(&u, &f, 4);
  u = u + 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

static void set_bf16(__nv_bfloat16 *dst, float v) {
  const uint16_t b = bf16_bits(v);
  memcpy(dst, &b, 2);
}

static void to_device_layout(const mcl_mlp &p, MlpDev &d) {
  memset(&d, 0, sizeof d);
  const float *f = reinterpret_cast<const float *>(&p);
  for (int n = 0; n < kH; n++) {
    for (int k = 0; k < kIn; k++) set_bf16(&d.w1[n][k], 0.5f * f[oW1 + n * kIn + k]);
    for (int k = 0; k < kH; k++) set_bf16(&d.w2[n][k], 0.5f * f[oW2 + n * kH + k]);
    d.b1[n] = 0.5f * f[oB1 + n];
    d.b2[n] = 0.5f * f[oB2 + n];
  }
  for (int n = 0; n < kOut; n++) {
    for (int k = 0; k < kH; k++) set_bf16(&d.w3[n][k], f[oW3 + n * kH + k]);
    d.b3[n] = f[oB3 + n];
  }
}

// ---- device helpers ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float sigm_f(float z) { return __fdividef(1.f, 1.f + __expf(-fmaxf(z, -80.f))); }
__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// SiLU of two halved pre-activations h = z / 2 (FP32), returned as packed BF16 (low half: the first):
// z sigmoid(z) = h + h tanh(h), with the hardware tanh approximation in FP32 and one paired FP32 fma, rounded once
// to BF16. Inference and training both use exactly this.
__device__ __forceinline__ float tanh_hw(float h) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
  return t;
}
__device__ __forceinline__ uint32_t silu2h(float h0, float h1) {
  const float2 h = make_float2(h0, h1);
  const float2 r = __ffma2_rn(h, make_float2(tanh_hw(h0), tanh_hw(h1)), h);
  return pack2(r.x, r.y);
}
__device__ __forceinline__ uint32_t silu2(float z0, float z1) { return silu2h(0.5f * z0, 0.5f * z1); }

// Four 8x8 BF16 matrices from shared memory; lane l gives the address of row l % 8 of matrix l / 8.
__device__ __forceinline__ void ldsm_x4(const void *row_addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"((unsigned)__cvta_generic_to_shared(row_addr)));
}
__device__ __forceinline__ float bf_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf_hi(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Features of a site from its neighbours (weights w in {0, 1}) and T.
__device__ __forceinline__ void site_features(const Vec3 (&nb)[6], const float (&w)[6], float T, float (&f)[kIn]) {
  float mxx = 0.f, mxy = 0.f, mxz = 0.f, myy = 0.f, myz = 0.f, mzz = 0.f, k = 0.f;
#pragma unroll
  for (int d = 0; d < 6; d++) {
    const float ax = w[d] * nb[d].x, ay = w[d] * nb[d].y, az = w[d] * nb[d].z;
    mxx = fmaf(ax, nb[d].x, mxx);
    mxy = fmaf(ax, nb[d].y, mxy);
    mxz = fmaf(ax, nb[d].z, mxz);
    myy = fmaf(ay, nb[d].y, myy);
    myz = fmaf(ay, nb[d].z, myz);
    mzz = fmaf(az, nb[d].z, mzz);
    k += w[d];
  }
  const float c = 1.f / 6.f;
  f[0] = fmaf(1.5f, mxx, -0.5f * k) * c;
  f[1] = 1.5f * mxy * c;
  f[2] = 1.5f * mxz * c;
  f[3] = fmaf(1.5f, myy, -0.5f * k) * c;
  f[4] = 1.5f * myz * c;
  f[5] = fmaf(1.5f, mzz, -0.5f * k) * c;
  f[6] = T;
}

// The MLP for the 32 sites of a warp (lane = site). All 32 lanes must call it (mma.sync is warp-wide). As / Out:
// this warp's scratch in shared memory.
__device__ __forceinline__ void warp_mlp(const MlpDev &S, __nv_bfloat16 (*As)[24], float (*Out)[4],
                                         const float (&f)[kIn], float (&o)[kOut]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // ldmatrix rows: lane l addresses row (l & 7) of matrix (l >> 3); matrices 0, 1 = k halves of n-tile A,
  // matrices 2, 3 = k halves of n-tile A + 1 (layers 1, 2) or of k-step + 1 (layer 3)
  const int lr = lane & 7, lm = lane >> 3;
  uint32_t *row = reinterpret_cast<uint32_t *>(As[lane]);
  row[0] = pack2(f[0], f[1]);
  row[1] = pack2(f[2], f[3]);
  row[2] = pack2(f[4], f[5]);
  row[3] = pack2(f[6], 0.f);
  row[4] = row[5] = row[6] = row[7] = 0u;
  __syncwarp();
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    const int r0 = 16 * mt + g, r1 = r0 + 8;
    const uint32_t a1[4] = {ld32(&As[r0][2 * t]), ld32(&As[r1][2 * t]), ld32(&As[r0][2 * t + 8]),
                            ld32(&As[r1][2 * t + 8])};
    uint32_t h1[4][4];
#pragma unroll
    for (int ks = 0; ks < 4; ks++) {  // n-tiles 2 ks, 2 ks + 1 of layer 1 = k-step ks of layer 2
      uint32_t bq[4];
      ldsm_x4(&S.w1[(2 * ks + (lm >> 1)) * 8 + lr][8 * (lm & 1)], bq[0], bq[1], bq[2], bq[3]);
      float c[2][4];
#pragma unroll
      for (int hh = 0; hh < 2; hh++) {
        const float2 bb = *reinterpret_cast<const float2 *>(&S.b1[(2 * ks + hh) * 8 + 2 * t]);
        c[hh][0] = c[hh][2] = bb.x;
        c[hh][1] = c[hh][3] = bb.y;
        mma_bf16(c[hh], a1, bq[2 * hh], bq[2 * hh + 1]);
      }
      h1[ks][0] = silu2h(c[0][0], c[0][1]);
      h1[ks][1] = silu2h(c[0][2], c[0][3]);
      h1[ks][2] = silu2h(c[1][0], c[1][1]);
      h1[ks][3] = silu2h(c[1][2], c[1][3]);
    }
    uint32_t h2[4][4];
#pragma unroll
    for (int ks2 = 0; ks2 < 4; ks2++) {
      float c[2][4];
#pragma unroll
      for (int hh = 0; hh < 2; hh++) {
        const float2 bb = *reinterpret_cast<const float2 *>(&S.b2[(2 * ks2 + hh) * 8 + 2 * t]);
        c[hh][0] = c[hh][2] = bb.x;
        c[hh][1] = c[hh][3] = bb.y;
      }
#pragma unroll
      for (int ks = 0; ks < 4; ks++) {
        uint32_t bq[4];
        ldsm_x4(&S.w2[(2 * ks2 + (lm >> 1)) * 8 + lr][16 * ks + 8 * (lm & 1)], bq[0], bq[1], bq[2], bq[3]);
        mma_bf16(c[0], h1[ks], bq[0], bq[1]);
        mma_bf16(c[1], h1[ks], bq[2], bq[3]);
      }
      h2[ks2][0] = silu2h(c[0][0], c[0][1]);
      h2[ks2][1] = silu2h(c[0][2], c[0][3]);
      h2[ks2][2] = silu2h(c[1][0], c[1][1]);
      h2[ks2][3] = silu2h(c[1][2], c[1][3]);
    }
    const float2 b3 = *reinterpret_cast<const float2 *>(&S.b3[2 * t]);
    float c3[4] = {b3.x, b3.y, b3.x, b3.y};
#pragma unroll
    for (int kp = 0; kp < 2; kp++) {  // k-steps 2 kp, 2 kp + 1
      uint32_t bq[4];
      ldsm_x4(&S.w3[lr][16 * (2 * kp + (lm >> 1)) + 8 * (lm & 1)], bq[0], bq[1], bq[2], bq[3]);
      mma_bf16(c3, h2[2 * kp], bq[0], bq[1]);
      mma_bf16(c3, h2[2 * kp + 1], bq[2], bq[3]);
    }
    if (t < 2) {
      *reinterpret_cast<float2 *>(&Out[r0][2 * t]) = make_float2(c3[0], c3[1]);
      *reinterpret_cast<float2 *>(&Out[r1][2 * t]) = make_float2(c3[2], c3[3]);
    }
  }
  __syncwarp();
  const float4 ov = *reinterpret_cast<const float4 *>(Out[lane]);
  o[0] = ov.x;
  o[1] = ov.y;
  o[2] = ov.z;
  o[3] = ov.w;
  __syncwarp();
}

// ---- the same network on tcgen05 (mlp_tc.cuh): a CTA of 256 threads, one row (site) per thread ---------------
// Bias + SiLU of 32 accumulator columns c0 .. c0 + 31 of this thread's row, packed to BF16 into its row of a
// K = 64 core-matrix tile.
__device__ __forceinline__ void tc_act_store(uint8_t *tile, int row, int c0, const float (&v)[32],
                                             const float *__restrict__ bias) {
#pragma unroll
  for (int ch = 0; ch < 4; ch++) {
    uint4 p;
    uint32_t *pp = reinterpret_cast<uint32_t *>(&p);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int c = 8 * ch + 2 * i;
      pp[i] = silu2h(v[c] + bias[c0 + c], v[c + 1] + bias[c0 + c + 1]);
    }
    *reinterpret_cast<uint4 *>(tile + core_off(row, c0 + 8 * ch, 64)) = p;
  }
}

// All 256 threads call it with their row's features; false (CTA-uniform) after a tensor-core timeout, in which case
// the caller frees the tensor memory (tc_teardown) and stops.
__device__ __forceinline__ bool cta_mlp_tc(TcSmem &S, unsigned &phase, long long timeout_ns, const float (&f)[kIn],
                                           float (&o)[kOut]) {
  const int tid = threadIdx.x, t = tid >> 7, row = tid & 127;
  uint8_t *a1 = S.a1 + t * kTcA1;
  uint4 lo;
  lo.x = pack2(f[0], f[1]);
  lo.y = pack2(f[2], f[3]);
  lo.z = pack2(f[4], f[5]);
  lo.w = pack2(f[6], 0.f);
  *reinterpret_cast<uint4 *>(a1 + core_off(row, 0, 16)) = lo;
  *reinterpret_cast<uint4 *>(a1 + core_off(row, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
  constexpr uint32_t id64 = tc_idesc(128, 64), id16 = tc_idesc(128, 16);
  if (!tc_stage(S, phase, timeout_ns, [&] {
        for (int tt = 0; tt < 2; tt++)
          tc_mma(S.tmem + tt * 64, tc_desc(S.a1 + tt * kTcA1, 128, 256), tc_desc(S.w1, 128, 256), id64, 0);
      }))
    return false;
  const uint32_t tcol = S.tmem + ((uint32_t)(32 * ((tid >> 5) & 3)) << 16) + t * 64;
  uint8_t *a2 = S.a2 + t * kTcA2;
#pragma unroll
  for (int hf = 0; hf < 2; hf++) {
    float v[32];
    tc_ld32(tcol + 32 * hf, v);
    tc_act_store(a2, row, 32 * hf, v, S.b1);
  }
  if (!tc_stage(S, phase, timeout_ns, [&] {
        for (int tt = 0; tt < 2; tt++)
          for (int ks = 0; ks < 4; ks++)
            tc_mma(S.tmem + tt * 64, tc_desc(S.a2 + tt * kTcA2 + ks * 256, 128, 1024),
                   tc_desc(S.w2 + ks * 256, 128, 1024), id64, ks > 0);
      }))
    return false;
#pragma unroll
  for (int hf = 0; hf < 2; hf++) {  // layer 2 has completed: its input tile may be overwritten with h2
    float v[32];
    tc_ld32(tcol + 32 * hf, v);
    tc_act_store(a2, row, 32 * hf, v, S.b2);
  }
  if (!tc_stage(S, phase, timeout_ns, [&] {
        for (int tt = 0; tt < 2; tt++)
          for (int ks = 0; ks < 4; ks++)
            tc_mma(S.tmem + tt * 64, tc_desc(S.a2 + tt * kTcA2 + ks * 256, 128, 1024),
                   tc_desc(S.w3 + ks * 256, 128, 1024), id16, ks > 0);
      }))
    return false;
  float v4[4];
  tc_ld4(tcol, v4);
#pragma unroll
  for (int k = 0; k < kOut; k++) o[k] = v4[k] + S.b3[k];
  return true;
}

// ---- the same network per warpgroup: 128 threads evaluate their own 128-row tile, independently of the CTA's
// other warpgroup (named barrier 1 + wg, their own commit mbarrier), so that one warpgroup's tensor-core round trips
// overlap the other's scalar work.
__device__ __forceinline__ void wg_bar(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory"); }

template <typename Issue>
__device__ __forceinline__ bool wg_stage(unsigned long long *bar, volatile int *wfail, unsigned &phase,
                                         long long timeout_ns, int wg, Issue issue) {
  tc_fence_async_smem();
  tc_fence_before();
  wg_bar(wg);
  if ((threadIdx.x & 127) == 0) {
    tc_fence_after();
    issue();
    tc_commit(bar);
  }
  const bool ok = tc_wait(bar, phase, timeout_ns);
  if (!ok) atomicOr((int *)wfail, 1);
  wg_bar(wg);
  if (*wfail) {  // wait (bounded) for the commit in flight before the tensor memory is freed
    tc_wait(bar, phase, timeout_ns);
    return false;
  }
  phase ^= 1u;
  tc_fence_after();
  return true;
}

// cta_mlp_tc for the warpgroup wg = threadIdx.x / 128 (tile wg, tensor-memory columns 64 wg .. 64 wg + 63); false
// (warpgroup-uniform) after a tensor-core timeout.
__device__ __forceinline__ bool wg_mlp_tc(TcSmem &S, unsigned long long *bar, volatile int *wfail, unsigned &phase,
                                          long long timeout_ns, const float (&f)[kIn], float (&o)[kOut]) {
  const int tid = threadIdx.x, wg = tid >> 7, row = tid & 127;
  uint8_t *a1 = S.a1 + wg * kTcA1;
  uint4 lo;
  lo.x = pack2(f[0], f[1]);
  lo.y = pack2(f[2], f[3]);
  lo.z = pack2(f[4], f[5]);
  lo.w = pack2(f[6], 0.f);
  *reinterpret_cast<uint4 *>(a1 + core_off(row, 0, 16)) = lo;
  *reinterpret_cast<uint4 *>(a1 + core_off(row, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
  constexpr uint32_t id64 = tc_idesc(128, 64), id16 = tc_idesc(128, 16);
  const uint32_t dcol = S.tmem + wg * 64;
  if (!wg_stage(bar, wfail, phase, timeout_ns, wg,
                [&] { tc_mma(dcol, tc_desc(a1, 128, 256), tc_desc(S.w1, 128, 256), id64, 0); }))
    return false;
  const uint32_t tcol = dcol + ((uint32_t)(32 * ((tid >> 5) & 3)) << 16);
  uint8_t *a2 = S.a2 + wg * kTcA2;
#pragma unroll
  for (int hf = 0; hf < 2; hf++) {
    float v[32];
    tc_ld32(tcol + 32 * hf, v);
    tc_act_store(a2, row, 32 * hf, v, S.b1);
  }
  if (!wg_stage(bar, wfail, phase, timeout_ns, wg, [&] {
        for (int ks = 0; ks < 4; ks++)
          tc_mma(dcol, tc_desc(a2 + ks * 256, 128, 1024), tc_desc(S.w2 + ks * 256, 128, 1024), id64, ks > 0);
      }))
    return false;
#pragma unroll
  for (int hf = 0; hf < 2; hf++) {  // layer 2 has completed: its input tile may be overwritten with h2
    float v[32];
    tc_ld32(tcol + 32 * hf, v);
    tc_act_store(a2, row, 32 * hf, v, S.b2);
  }
  if (!wg_stage(bar, wfail, phase, timeout_ns, wg, [&] {
        for (int ks = 0; ks < 4; ks++)
          tc_mma(dcol, tc_desc(a2 + ks * 256, 128, 1024), tc_desc(S.w3 + ks * 256, 128, 1024), id16, ks > 0);
      }))
    return false;
  float v4[4];
  tc_ld4(tcol, v4);
#pragma unroll
  for (int k = 0; k < kOut; k++) o[k] = v4[k] + S.b3[k];
  return true;
}

// Network outputs of feature rows on tcgen05 (the same outputs as k_mlp_forward).
__global__ void __launch_bounds__(kTcRows) k_mlp_forward_tc(const MlpTC *__restrict__ w,
                                                            const float *__restrict__ feat, long long n,
                                                            float *__restrict__ out, unsigned *__restrict__ err,
                                                            long long timeout_ns) {
  extern __shared__ __align__(128) unsigned char tc_dyn[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(tc_align128(tc_dyn));
  tc_setup(S, w);
  unsigned phase = 0;
  for (long long base = (long long)blockIdx.x * kTcRows; base < n; base += (long long)gridDim.x * kTcRows) {
    const long long i = base + threadIdx.x;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; k++) f[k] = i < n ? feat[i * kFeat + k] : 0.f;
    float o[kOut];
    if (!cta_mlp_tc(S, phase, timeout_ns, f, o)) {
      if (threadIdx.x == 0) atomicOr(err, 1u);
      break;
    }
    if (i < n)
#pragma unroll
      for (int k = 0; k < kOut; k++) out[i * kOut + k] = o[k];
  }
  tc_teardown(S);
}

static void to_tc_layout(const mcl_mlp &p, MlpTC &d) {
  memset(&d, 0, sizeof d);
  const float *f = reinterpret_cast<const float *>(&p);
  for (int n = 0; n < kH; n++) {
    for (int k = 0; k < kIn; k++) {
      const uint16_t b = bf16_bits(0.5f * f[oW1 + n * kIn + k]);
      memcpy(d.w1 + core_off(n, k, 16), &b, 2);
    }
    for (int k = 0; k < kH; k++) {
      const uint16_t b = bf16_bits(0.5f * f[oW2 + n * kH + k]);
      memcpy(d.w2 + core_off(n, k, 64), &b, 2);
    }
    d.b1[n] = 0.5f * f[oB1 + n];
    d.b2[n] = 0.5f * f[oB2 + n];
  }
  for (int n = 0; n < kOut; n++) {
    for (int k = 0; k < kH; k++) {
      const uint16_t b = bf16_bits(f[oW3 + n * kH + k]);
      memcpy(d.w3 + core_off(n, k, 64), &b, 2);
    }
    d.b3[n] = f[oB3 + n];
  }
}

struct Head {
  Vec3 mu;
  float kappa;
};

__device__ __forceinline__ Head mlp_head(const float (&o)[kOut], float kappa_max) {
  Head h;
  const float na = sqrtf(fmaf(o[0], o[0], fmaf(o[1], o[1], o[2] * o[2])));
  if (na > 1e-12f) {
    const float inv = 1.f / na;
    h.mu = Vec3{o[0] * inv, o[1] * inv, o[2] * inv};
  } else {
    h.mu = Vec3{0.f, 0.f, 1.f};
  }
  const float kr = o[3] > 20.f ? o[3] : log1pf(expf(o[3]));
  h.kappa = fminf(fmaxf(kr, kKappaMin), kappa_max);
  return h;
}

// 4 pi q(n) of the mixture at t = mu.n: 0.95 g + 0.05 with g = kappa cosh(kappa t) / sinh(kappa)
// = kappa (e^{kappa (|t| - 1)} + e^{-kappa (|t| + 1)}) / (1 - e^{-2 kappa}); inv_den = 1 / (1 - e^{-2 kappa}),
// e2k = e^{-2 kappa}. One exponential: the second term is e2k / the first. e2k comes from its own exponential, not
// from 1 + expm1(-2 kappa): that sum cancels in FP32 (all of e^{-2 kappa} is lost for kappa > 8.7), which would drop
// the second term, make q wrong by up to a few per cent for directors nearly perpendicular to mu, and bias the chain
// toward them wherever the network's kappa lies between a few and a few tens.
__device__ __forceinline__ float q4pi(float t, float kappa, float inv_den, float e2k) {
  const float e1 = __expf(kappa * (fabsf(t) - 1.f));
  const float e2 = e1 > 1e-30f ? __fdividef(e2k, e1) : 0.f;
  return fmaf(1.f - kEps, kappa * (e1 + e2) * inv_den, kEps);
}

// A draw from the mixture: u_mix < 0.05 uniform on the sphere, else the vMF about mu by Wood's method with a
// random sign (em1 = expm1(-2 kappa)).
__device__ __forceinline__ Vec3 sample_proposal(const Head &h, float em1, float e2k, float u_mix, float u_w,
                                                float u_phi, bool neg) {
  const bool uni = u_mix < kEps;
  float w, r;
  Vec3 base;
  if (uni) {
    w = fmaf(2.f, u_w, -1.f);  // exact, and so are 1 - w and 1 + w
    r = sqrtf(fmaxf(0.f, (1.f - w) * (1.f + w)));
    base = Vec3{0.f, 0.f, 1.f};
  } else {
    // s = 1 - w = -log(1 + x) / kappa with x = (1 - u) em1 (em1 = e^{-2 kappa} - 1): as log1p(x) while 1 + x is
    // at least 1/2, and as log(u + (1 - u) e^{-2 kappa}) below, where e^{-2 kappa} (e2k) would vanish next to 1 in em1;
    // the tangential part from s (2 - s): near mu, 1 - w is a few ulps of 1 in FP32 and 1 - w^2 would lose its digits
    const float x = (1.f - u_w) * em1;
    const float lg = x >= -0.5f ? log1pf(x) : logf(fmaf(1.f - u_w, e2k, u_w));
    const float sw = fminf(fmaxf(-lg / h.kappa, 0.f), 2.f);
    w = 1.f - sw;
    r = sqrtf(sw * (2.f - sw));
    base = h.mu;
  }
  // orthonormal e1, e2 perpendicular to base: e1 = base x (x or y axis), e2 = base x e1
  Vec3 e1 = fabsf(base.x) < 0.9f ? Vec3{0.f, base.z, -base.y} : Vec3{-base.z, 0.f, base.x};
  const float i1 = rsqrtf(dot(e1, e1));
  e1 = Vec3{e1.x * i1, e1.y * i1, e1.z * i1};
  const Vec3 e2{base.y * e1.z - base.z * e1.y, base.z * e1.x - base.x * e1.z, base.x * e1.y - base.y * e1.x};
  float sp, cp;
  sincospif(2.f * u_phi, &sp, &cp);
  Vec3 v{fmaf(w, base.x, r * fmaf(cp, e1.x, sp * e2.x)), fmaf(w, base.y, r * fmaf(cp, e1.y, sp * e2.y)),
         fmaf(w, base.z, r * fmaf(cp, e1.z, sp * e2.z))};
  const float inv = rsqrtf(dot(v, v));
  const float sgn = (neg && !uni) ? -inv : inv;
  return Vec3{v.x * sgn, v.y * sgn, v.z * sgn};
}

__device__ __forceinline__ float u24(uint32_t v) { return (float)(v >> 8) * 0x1p-24f; }

// ---- the learned sweep: one colour, one thread per site ----------------------------------------------------------
// TC: the network on tcgen05 (a CTA-wide pass over its 256 sites) instead of mma.sync warps. Dynamic shared memory:
// TcSmem (TC) or the warp path's weights and scratch.
constexpr size_t kWarpMlpSmem = sizeof(MlpDev) + sizeof(__nv_bfloat16) * (kThreads / 32) * 32 * 24 +
                                sizeof(float) * (kThreads / 32) * 32 * 4 + 128;
constexpr size_t kTcMlpSmem = sizeof(TcSmem) + 128;

template <int POT, int GEO, bool TC>
__global__ void __launch_bounds__(kThreads, 3) k_sweep_learned(ModelDev m, const RepDesc *__restrict__ reps,
                                                            RepState *__restrict__ st, float *__restrict__ dir,
                                                            const uint8_t *__restrict__ pt,
                                                            const float *__restrict__ nrm,
                                                            const unsigned long long *__restrict__ sweep_ctr,
                                                            int colour, const int *__restrict__ blk_rep,
                                                            const long long *__restrict__ blk_base, int n_blocks,
                                                            const MlpDev *__restrict__ mlp,
                                                            const MlpTC *__restrict__ mlp_tc,
                                                            unsigned *__restrict__ err, float kappa_max,
                                                            int measure, double *__restrict__ partials) {
  extern __shared__ __align__(128) unsigned char ls_dyn[];
  __shared__ double red[kThreads / 32][kPartials];
  unsigned char *sbase = tc_align128(ls_dyn);
  MlpDev *S = nullptr;
  __nv_bfloat16(*As)[32][24] = nullptr;
  float(*Out)[32][4] = nullptr;
  TcSmem *T = nullptr;
  unsigned phase = 0;
  if constexpr (TC) {
    T = reinterpret_cast<TcSmem *>(sbase);
    tc_setup(*T, mlp_tc);
  } else {
    S = reinterpret_cast<MlpDev *>(sbase);
    As = reinterpret_cast<__nv_bfloat16(*)[32][24]>(sbase + sizeof(MlpDev));
    Out = reinterpret_cast<float(*)[32][4]>(sbase + sizeof(MlpDev) +
                                            sizeof(__nv_bfloat16) * (kThreads / 32) * 32 * 24);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpDev) / 16); i += blockDim.x)
      reinterpret_cast<uint4 *>(S)[i] = reinterpret_cast<const uint4 *>(mlp)[i];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5;
  const unsigned long long sweep = *sweep_ctr;
  for (int b = blockIdx.x; b < n_blocks; b += gridDim.x) {
    const int rep = blk_rep[b];
    const RepDesc R = reps[rep];
    const RepState St = st[rep];
    const long long q = blk_base[b] + threadIdx.x;
    const int hx = (R.nx + 1) >> 1;
    const long long total = (long long)hx * R.ny * R.nz;
    bool valid = false;
    int x = 0, y = 0, z = 0, sid = -1;
    Vec3 n{0.f, 0.f, 1.f}, s{0.f, 0.f, 0.f};
    Vec3 nb[6];
    float w[6];
#pragma unroll
    for (int d = 0; d < 6; d++) {
      nb[d] = Vec3{0.f, 0.f, 0.f};
      w[d] = 0.f;
    }
    if (q < total) {  // a replica has fewer than 2^32 sites (checked at creation): 32-bit decode
      const unsigned qq = (unsigned)q, row = qq / (unsigned)hx;
      const int xh = (int)(qq - row * (unsigned)hx);
      z = (int)(row / (unsigned)R.ny);
      y = (int)(row - (unsigned)z * (unsigned)R.ny);
      x = 2 * xh + ((colour + y + z) & 1);
      if (x < R.nx) valid = gather_site_rows<GEO>(R, dir, pt, nrm, x, y, z, n, nb, w, sid, s);
    }
    float f[kIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (valid) site_features(nb, w, St.T, f);
    float o[kOut];
    if constexpr (TC) {
      if (!cta_mlp_tc(*T, phase, 2000000000ll, f, o)) {  // CTA-uniform: stop, report, free the tensor memory
        if (threadIdx.x == 0) atomicOr(err, 1u);
        break;
      }
    } else {
      warp_mlp(*S, As[warp], Out[warp], f, o);
    }
    unsigned accepted = 0;
    float ob[kPartials] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (valid) {
      const Head h = mlp_head(o, kappa_max);
      const U4 u = site_draws(R.seed, sweep, (uint32_t)site_linear(R, x, y, z), 1);
      const float em1 = expm1f(-2.f * h.kappa), e2k = expf(-2.f * h.kappa);
      const Vec3 nn = sample_proposal(h, em1, e2k, u24(u.x), u24(u.y), u24(u.z), (u.x & 1u) != 0u);
      float b_old, b_new;
      bond_sum2<POT, false, true, float>(m, n, nn, nb, w, b_old, b_new);
      const float s_old = single_energy<true>(m, n, sid, s, St.elecE), s_new = single_energy<true>(m, nn, sid, s, St.elecE);
      const float e_old = __fadd_rn(b_old, s_old);
      const float e_new = __fadd_rn(b_new, s_new);
      const float dE = __fadd_rn(e_new, -e_old);
      bool acc;
      if (St.T > 0.f) {  // u < e^{-dE/T} q(n) / q(n'), without logarithms
        const float inv_den = -1.f / em1;
        const float q_old = q4pi(dot(h.mu, n), h.kappa, inv_den, e2k), q_new = q4pi(dot(h.mu, nn), h.kappa, inv_den, e2k);
        acc = u24(u.w) * q_new < __expf(-dE / St.T) * q_old;
      } else {
        acc = dE <= 0.f;
      }
      if (acc) {
        dir[dir_index(R, 0, x, y, z)] = nn.x;
        dir[dir_index(R, 1, x, y, z)] = nn.y;
        dir[dir_index(R, 2, x, y, z)] = nn.z;
        accepted = 1;
      }
      if (measure) {  // the site is final: colour 0 adds its single-site terms, colour 1 2 bond + single
        const Vec3 nf = acc ? nn : n;
        const float bf = acc ? b_new : b_old, sf = acc ? s_new : s_old;
        ob[0] = colour == 0 ? sf : __fadd_rn(__fmul_rn(2.f, bf), sf);
        ob[1] = fmaf(1.5f * nf.x, nf.x, -0.5f);
        ob[2] = 1.5f * nf.x * nf.y;
        ob[3] = 1.5f * nf.x * nf.z;
        ob[4] = fmaf(1.5f * nf.y, nf.y, -0.5f);
        ob[5] = 1.5f * nf.y * nf.z;
        ob[6] = fmaf(1.5f * nf.z, nf.z, -0.5f);
        ob[7] = nf.x;
        ob[8] = nf.y;
        ob[9] = nf.z;
      }
    }
    const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(&st[rep].acc, (unsigned long long)wsum);
    if (measure) {  // uniform: table entry b is this block's alone, in both colour launches. FP32 per-site terms
                    // summed in FP32 over a warp (32 sites), then in FP64.
#pragma unroll
      for (int k = 0; k < kPartials; k++) {
        float v = ob[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) red[warp][k] = (double)v;
      }
      __syncthreads();
      if (threadIdx.x < kPartials) {
        double v = 0.0;
        for (int w2 = 0; w2 < kThreads / 32; w2++) v += red[w2][threadIdx.x];
        double *dst = partials + (long long)b * kPartials + threadIdx.x;
        *dst = colour == 0 ? v : *dst + v;
      }
      __syncthreads();
    }
  }
  if constexpr (TC) tc_teardown(*T);
}

// Network outputs (before the head) for feature rows, for parity tests of the tensor-core path.
__global__ void __launch_bounds__(kThreads) k_mlp_forward(const MlpDev *__restrict__ mlp,
                                                          const float *__restrict__ feat, long long n,
                                                          float *__restrict__ out) {
  __shared__ __align__(16) MlpDev S;
  __shared__ __align__(16) __nv_bfloat16 As[kThreads / 32][32][24];
  __shared__ __align__(16) float Out[kThreads / 32][32][4];
  for (int i = threadIdx.x; i < (int)(sizeof(MlpDev) / 16); i += blockDim.x)
    reinterpret_cast<uint4 *>(&S)[i] = reinterpret_cast<const uint4 *>(mlp)[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  for (long long base = (long long)blockIdx.x * kThreads; base < n; base += (long long)gridDim.x * kThreads) {
    const long long i = base + threadIdx.x;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; k++) f[k] = i < n ? feat[i * kFeat + k] : 0.f;
    float o[kOut];
    warp_mlp(S, As[warp], Out[warp], f, o);
    if (i < n)
#pragma unroll
      for (int k = 0; k < kOut; k++) out[i * kOut + k] = o[k];
  }
}

// Training samples: n sites of one replica drawn with Philox(seed, sample index), their features and directors.
template <int GEO>
__global__ void k_extract_samples(const RepDesc *__restrict__ reps, const RepState *__restrict__ st,
                                  const float *__restrict__ dir, const uint8_t *__restrict__ pt,
                                  const float *__restrict__ nrm, int rep, long long n, unsigned long long seed,
                                  float *__restrict__ feat, float *__restrict__ dirs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDesc R = reps[rep];
  const U4 u = stream_draws((uint32_t)i, (uint32_t)(i >> 32), seed, 0u, 3u);
  const unsigned long long N = (unsigned long long)R.nx * R.ny * R.nz;
  const unsigned long long site = (((unsigned long long)u.x << 32) | u.y) % N;
  const int x = (int)(site % R.nx);
  const unsigned long long row = site / R.nx;
  const int y = (int)(row % R.ny), z = (int)(row / R.ny);
  Vec3 nv, nb[6], s;
  float w[6];
  int sid;
  float f[kIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const bool valid = gather_site_rows<GEO>(R, dir, pt, nrm, x, y, z, nv, nb, w, sid, s);
  if (valid) site_features(nb, w, st[rep].T, f);
#pragma unroll
  for (int k = 0; k < kIn; k++) feat[i * kFeat + k] = f[k];
  feat[i * kFeat + 7] = valid ? 1.f : 0.f;
  dirs[i * 3 + 0] = valid ? nv.x : 0.f;
  dirs[i * 3 + 1] = valid ? nv.y : 0.f;
  dirs[i * 3 + 2] = valid ? nv.z : 0.f;
}

// ---- training ------------------------------------------------------------------------------------------------
constexpr int kTB = 64;            // samples (threads) per training block
constexpr int kHP = kH + 1;        // row pitch of the per-sample activation arrays
constexpr int kWPad = kNP + 4;     // BF16-rounded weights in shared memory
constexpr size_t kTrainSmem = sizeof(float) * (kWPad + kTB * 9 + 4 * kTB * kHP + kTB * 5 + kTB);

// Forward and backward pass of kTB samples (one per thread) with the pass copy wr of the parameters; writes this block's
// parameter gradient of the mean loss (scale = 1 / batch) and its loss sum to partial[blockIdx.x][0 .. kNP].
__global__ void __launch_bounds__(kTB) k_mlp_grad(const float *__restrict__ wr, const float *__restrict__ feat,
                                                  const float *__restrict__ dirs, long long n, float kappa_max,
                                                  float scale, float *__restrict__ partial) {
  extern __shared__ float sm[];
  float *W = sm;
  float *X = W + kWPad;            // [kTB][9]
  float *H1 = X + kTB * 9;         // [kTB][kHP]
  float *H2 = H1 + kTB * kHP;
  float *DZ1 = H2 + kTB * kHP;
  float *DZ2 = DZ1 + kTB * kHP;
  float *DO = DZ2 + kTB * kHP;     // [kTB][5]
  float *LS = DO + kTB * 5;        // [kTB]
  const int tid = threadIdx.x;
  for (int i = tid; i < kNP; i += kTB) W[i] = wr[i];
  __syncthreads();
  const long long s = (long long)blockIdx.x * kTB + tid;
  const bool valid = s < n && feat[s * kFeat + 7] != 0.f;
  float x[kIn];
#pragma unroll
  for (int k = 0; k < kIn; k++) {
    x[k] = valid ? bf16r(feat[s * kFeat + k]) : 0.f;
    X[tid * 9 + k] = x[k];
  }
  float z1[kH], h1[kH];
#pragma unroll 4
  for (int j = 0; j < kH; j += 2) {
    float a0 = W[oB1 + j], a1 = W[oB1 + j + 1];
#pragma unroll
    for (int k = 0; k < kIn; k++) {
      a0 = fmaf(W[oW1 + j * kIn + k], x[k], a0);
      a1 = fmaf(W[oW1 + (j + 1) * kIn + k], x[k], a1);
    }
    z1[j] = a0;
    z1[j + 1] = a1;
    const uint32_t hv = silu2(a0, a1);
    h1[j] = bf_lo(hv);
    h1[j + 1] = bf_hi(hv);
    H1[tid * kHP + j] = h1[j];
    H1[tid * kHP + j + 1] = h1[j + 1];
  }
  float z2[kH], h2[kH];
#pragma unroll 2
  for (int j = 0; j < kH; j += 2) {
    float a0 = W[oB2 + j], a1 = W[oB2 + j + 1];
#pragma unroll
    for (int i = 0; i < kH; i++) {
      a0 = fmaf(W[oW2 + j * kH + i], h1[i], a0);
      a1 = fmaf(W[oW2 + (j + 1) * kH + i], h1[i], a1);
    }
    z2[j] = a0;
    z2[j + 1] = a1;
    const uint32_t hv = silu2(a0, a1);
    h2[j] = bf_lo(hv);
    h2[j + 1] = bf_hi(hv);
    H2[tid * kHP + j] = h2[j];
    H2[tid * kHP + j + 1] = h2[j + 1];
  }
  float o[kOut];
#pragma unroll
  for (int mo = 0; mo < kOut; mo++) {
    float a = W[oB3 + mo];
#pragma unroll
    for (int j = 0; j < kH; j++) a = fmaf(W[oW3 + mo * kH + j], h2[j], a);
    o[mo] = a;
  }
  // head, loss and d loss / d o
  float dout[kOut] = {0.f, 0.f, 0.f, 0.f};
  float loss = 0.f;
  if (valid) {
    const float nx = dirs[s * 3], ny = dirs[s * 3 + 1], nz = dirs[s * 3 + 2];
    const float na = sqrtf(fmaf(o[0], o[0], fmaf(o[1], o[1], o[2] * o[2])));
    const float inv = 1.f / fmaxf(na, 1e-20f);
    const float mx = o[0] * inv, my = o[1] * inv, mz = o[2] * inv;
    const float kr = o[3] > 20.f ? o[3] : log1pf(expf(o[3]));
    const float kappa = fminf(fmaxf(kr, kKappaMin), kappa_max);
    const float t = fmaf(mx, nx, fmaf(my, ny, mz * nz));
    const float at = fabsf(t);
    const float g = kappa * (expf(kappa * (at - 1.f)) + expf(-kappa * (at + 1.f))) / (-expm1f(-2.f * kappa));
    const float den = fmaf(1.f - kEps, g, kEps);
    loss = -logf(den);
    const float th = tanhf(kappa * t);
    const float dt = -(1.f - kEps) * g * kappa * th / den;
    const float ikc = kappa < 0.1f ? kappa * (-1.f / 3.f + kappa * kappa / 45.f) : 1.f / kappa - 1.f / tanhf(kappa);
    float dk = -(1.f - kEps) * g * (ikc + t * th) / den;
    if (!(kr > kKappaMin && kr < kappa_max)) dk = 0.f;
    dout[0] = scale * dt * (nx - t * mx) * inv;
    dout[1] = scale * dt * (ny - t * my) * inv;
    dout[2] = scale * dt * (nz - t * mz) * inv;
    dout[3] = scale * dk * sigm_f(o[3]);
  }
  LS[tid] = loss;
#pragma unroll
  for (int mo = 0; mo < kOut; mo++) DO[tid * 5 + mo] = dout[mo];
  // backward to the hidden layers (z2 is overwritten with dz2)
#pragma unroll 4
  for (int j = 0; j < kH; j++) {
    float a = 0.f;
#pragma unroll
    for (int mo = 0; mo < kOut; mo++) a = fmaf(W[oW3 + mo * kH + j], dout[mo], a);
    const float sg = sigm_f(z2[j]);
    z2[j] = a * sg * fmaf(z2[j], 1.f - sg, 1.f);
    DZ2[tid * kHP + j] = z2[j];
  }
#pragma unroll 4
  for (int i = 0; i < kH; i++) {
    float a = 0.f;
#pragma unroll
    for (int j = 0; j < kH; j++) a = fmaf(W[oW2 + j * kH + i], z2[j], a);
    const float sg = sigm_f(z1[i]);
    DZ1[tid * kHP + i] = a * sg * fmaf(z1[i], 1.f - sg, 1.f);
  }
  __syncthreads();
  // this block's weight gradients: thread tid owns column tid of every [out][in] matrix it can
  float *P = partial + (size_t)blockIdx.x * (kNP + 1);
  for (int r = 0; r < kH; r++) {  // w2[r][tid] = sum_s dz2[s][r] h1[s][tid]
    float a = 0.f;
    for (int q = 0; q < kTB; q++) a = fmaf(DZ2[q * kHP + r], H1[q * kHP + tid], a);
    P[oW2 + r * kH + tid] = a;
  }
  {
    float a[kIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, b1 = 0.f, b2 = 0.f;
    for (int q = 0; q < kTB; q++) {
      const float d1 = DZ1[q * kHP + tid];
#pragma unroll
      for (int k = 0; k < kIn; k++) a[k] = fmaf(d1, X[q * 9 + k], a[k]);
      b1 += d1;
      b2 += DZ2[q * kHP + tid];
    }
#pragma unroll
    for (int k = 0; k < kIn; k++) P[oW1 + tid * kIn + k] = a[k];
    P[oB1 + tid] = b1;
    P[oB2 + tid] = b2;
  }
#pragma unroll
  for (int mo = 0; mo < kOut; mo++) {  // w3[mo][tid]
    float a = 0.f;
    for (int q = 0; q < kTB; q++) a = fmaf(DO[q * 5 + mo], H2[q * kHP + tid], a);
    P[oW3 + mo * kH + tid] = a;
  }
  if (tid < kOut) {
    float a = 0.f;
    for (int q = 0; q < kTB; q++) a += DO[q * 5 + tid];
    P[oB3 + tid] = a;
  }
  if (tid == 0) {
    float a = 0.f;
    for (int q = 0; q < kTB; q++) a += LS[q];
    P[kNP] = a;
  }
}

// Fixed-order FP64 sum of the block partials: gradient (and loss sum in out[kNP]).
__global__ void k_grad_reduce(const float *__restrict__ partial, int nb, double *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kNP) return;
  double a = 0.0;
  for (int b = 0; b < nb; b++) a += (double)partial[(size_t)b * (kNP + 1) + p];
  out[p] = a;
}

// Biases stay FP32 in every pass (as in inference); weights are rounded to BF16.
__device__ __forceinline__ float pass_value(int p, float v) {
  const bool bias = (p >= oB1 && p < oB1 + kH) || (p >= oB2 && p < oB2 + kH) || p >= oB3;
  return bias ? v : bf16r(v);
}

// Adam on the FP32 master parameters, then their copy for the next forward pass (weights BF16-rounded).
__global__ void k_adam(const double *__restrict__ grad, float *__restrict__ params, float *__restrict__ wr,
                       float *__restrict__ m1, float *__restrict__ m2, float lr, float bc1, float bc2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  const float g = (float)grad[p];
  const float a = fmaf(0.9f, m1[p], 0.1f * g), b = fmaf(0.999f, m2[p], 0.001f * g * g);
  m1[p] = a;
  m2[p] = b;
  const float v = params[p] - lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
  params[p] = v;
  wr[p] = pass_value(p, v);
}

__global__ void k_round(const float *__restrict__ params, float *__restrict__ wr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kNP) wr[p] = pass_value(p, params[p]);
}

// ---- the learned sweep as colour passes on TMA-streamed planes (bulk and slab, tcgen05) -------------------------
// The plain colour pass (sweep_pass.cuh) with the learned proposal: work item = (replica, 64 x 8 tile, z segment);
// per plane the tile holds exactly 256 sites of the colour, one per thread (warp w: row y0 + w, all of one x
// parity), so each plane step is one 256-row tcgen05 MLP batch (cta_mlp_tc). Neighbours come from the plane
// window in shared memory (4 slots, two planes in flight, the -z neighbour carried from the step before), the
// update is written in place with the ghost copies of edge sites, and every per-site computation is the one
// k_sweep_learned makes (features, network, head, stream-1 draws, proposal, energies, Hastings test), so the two
// kernels take the same decisions. Waits are bounded: a plane that does not arrive sets bit 1 of the error word, a
// tensor-core stage bit 0; either way the CTA drains its copies, frees its tensor memory and returns.
struct LearnedPassArgs {
  const CUtensorMap *tmaps;
  float *dir;  // the buffer read and written (in place)
  const RepDesc *reps;
  RepState *st;
  const FusedItem *items;
  double *partials;  // [item][kPartials]: colour 0 writes, colour 1 adds
  const unsigned long long *sweep_ctr;
  const MlpTC *mlp_tc;
  unsigned *err;
  float kappa_max;
  int cur, colour, measure;
  long long timeout_ns;
};

constexpr int kLTY = 8, kLH = kLTY + 2, kLPF = RW * kLH, kLSlot = (3 * kLPF + 31) / 32 * 32, kLNS = 4;
// plane slots, their full and empty barriers, the tcgen05 operands
constexpr size_t kLearnedPassSmem = 128 + (size_t)kLNS * kLSlot * 4 + 2 * kLNS * 8 + sizeof(TcSmem) + 128;

// Ghost copies of one updated site (half index j of the half-row row0 of parity h, component 0): along a periodic
// y the site again at rows y + ny (y < 2) and y - ny (y >= ny - 2); along a periodic x, on each of those rows, half
// index nx / 2 for half index 0 and half index -1 for nx / 2 - 1.
static __device__ __noinline__ void learned_ghosts(float *row0, long long cs, int px, float vx, float vy, float vz,
                                                   int j, int nx, int ny, int y, bool perx, bool pery) {
  const float v[3] = {vx, vy, vz};
  for (int iy = 0; iy < 3; iy++) {
    if (iy == 1 && !(pery && y < 2)) continue;
    if (iy == 2 && !(pery && y >= ny - 2)) continue;
    float *rowp = row0 + (long long)(iy == 0 ? 0 : (iy == 1 ? ny : -ny)) * px;
    if (iy > 0)
      for (int q = 0; q < 3; q++) rowp[q * cs + j] = v[q];
    if (perx && j == 0)
      for (int q = 0; q < 3; q++) rowp[q * cs + (nx >> 1)] = v[q];
    if (perx && j == (nx >> 1) - 1)
      for (int q = 0; q < 3; q++) rowp[q * cs - 1] = v[q];
  }
}

// The two warpgroups (tile rows 0-3 and 4-7) run decoupled: each waits for the planes itself, evaluates its
// 128-row tile on the tensor cores with its own barriers, and every warp releases a plane slot (empty barrier) once
// it has loaded its neighbours from it; thread 0 refills a slot only after all eight warps released it. A warpgroup
// may run up to a plane ahead of the other, so one's tensor-core round trips overlap the other's scalar work.
template <int POT, int GEO>
__global__ void __launch_bounds__(kThreads, 2) k_learned_pass(ModelDev m, LearnedPassArgs a) {
  static_assert(kThreads == 32 * kLTY, "one warp per tile row, one site per thread");
  static_assert(kThreads == 2 * 128, "two warpgroups, one 128-row tile each");
  extern __shared__ __align__(128) unsigned char lp_dyn[];
  unsigned char *smem_raw = smem_align128(lp_dyn);
  float *slots = reinterpret_cast<float *>(smem_raw);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw + (size_t)kLNS * kLSlot * 4);
  unsigned long long *ebars = bars + kLNS;  // slot released by all eight warps
  TcSmem &T = *reinterpret_cast<TcSmem *>(tc_align128(smem_raw + (size_t)kLNS * kLSlot * 4 + 2 * kLNS * 8));
  __shared__ unsigned long long s_mma[2];  // tensor-core commits, one barrier per warpgroup
  __shared__ int s_wfail[2];               // per warpgroup: bit 0 a tensor-core wait, bit 1 a plane wait timed out
  __shared__ double red[kThreads / 32][kPartials];
  const FusedItem it = a.items[blockIdx.x];
  const RepDesc R = a.reps[it.rep];
  const RepState St = a.st[it.rep];
  const int tid = threadIdx.x;
  const CUtensorMap *map = a.tmaps + 2 * it.rep + a.cur;
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  const bool perx = R.periodic[0], pery = R.periodic[1], perz = R.periodic[2];
  const int x0 = it.x0, y0 = it.y0, z0 = it.z0, z1 = it.z1, j0 = x0 >> 1;
  const int colour = a.colour;
  const bool measure = a.measure != 0;
  const unsigned long long sweep = *a.sweep_ctr;
  constexpr unsigned box_bytes = 3u * kLPF * 4u;
  if (tid == 0) {
    s_wfail[0] = s_wfail[1] = 0;
    for (int q = 0; q < kLNS; q++) {
      mbar_init(&bars[q], 1);
      mbar_init(&ebars[q], kThreads / 32);
    }
    mbar_init(&s_mma[0], 1);
    mbar_init(&s_mma[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
  }
  tc_setup(T, a.mlp_tc);  // ends with a CTA barrier: the plane barriers are initialised for every thread
  const int wg = tid >> 7, lane = tid & 31;
  volatile int *wfail = &s_wfail[wg];
  unsigned phase = 0;

  const int pbeg = z0 - 1, pend = z1;
  auto plane_exists = [&](int p) { return perz || (p >= 0 && p < nz); };
  auto wrapz = [&](int p) { return p < 0 ? p + nz : (p >= nz ? p - nz : p); };
  auto slot_ptr = [&](int p) -> float * { return slots + (size_t)((unsigned)(p - pbeg) % kLNS) * kLSlot; };
  int last_issued = pbeg - 1;
  auto issue = [&](int p) -> bool {  // thread 0 only; false if the slot was not released in time
    if (p > pend) return true;
    const int lp = p - pbeg;
    const unsigned sl = (unsigned)lp % kLNS;
    if (lp >= kLNS && !mbar_wait_bounded(&ebars[sl], ((unsigned)lp / kLNS - 1u) & 1u, a.timeout_ns)) return false;
    last_issued = p;
    unsigned long long *bar = &bars[sl];
    if (!plane_exists(p)) {
      mbar_arrive(bar);
      return true;
    }
    mbar_expect_tx(bar, box_bytes);
    tma_load_plane(slot_ptr(p), map, j0, y0 - 1 + GY, wrapz(p), bar);
    return true;
  };
  auto release = [&](int p) {  // this warp has loaded what it needs from plane p
    __syncwarp();
    if (lane == 0) mbar_arrive(&ebars[(unsigned)(p - pbeg) % kLNS]);
  };
  int waited = pbeg - 1;
  bool pfail = false;  // thread 0: a slot was not released in time (published before its next plane barrier)
  // Flags are written only before a warpgroup barrier that precedes their reads, so every thread of the warpgroup
  // reads the same value.
  auto wait_plane = [&](int p) -> bool {  // warpgroup-uniform result
    if (p <= pend && p > waited) {
      const int lp = p - pbeg;
      if (plane_exists(p) && !mbar_wait_bounded(&bars[(unsigned)lp % kLNS], ((unsigned)lp / kLNS) & 1u, a.timeout_ns))
        atomicOr((int *)wfail, 2);
    }
    if (pfail) atomicOr((int *)wfail, 2);
    wg_bar(wg);
    if (*wfail) return false;
    if (p > waited) waited = p;
    return true;
  };
  if (tid == 0)
    for (int p = pbeg; p <= pbeg + kLNS - 1; p++) issue(p);

  const int r = tid >> 5, s = tid & 31;  // row y0 + r, half-row cell j0 + s
  const int y = y0 + r, jb = 4 + s, j = j0 + s;
  const bool live_row = y < ny;
  const long long cs = R.comp;
  unsigned accepted = 0;
  double dacc[kPartials];
#pragma unroll
  for (int q = 0; q < kPartials; q++) dacc[q] = 0.0;
  bool ok = wait_plane(z0 - 1) && wait_plane(z0);
  Vec3 pd{0.f, 0.f, 0.f};  // -z neighbour: plane k - 1, cell jb, this step's parity
  if (ok) {
    if (plane_exists(z0 - 1)) {
      const float *q0 = slot_ptr(z0 - 1) + ((r + 1) * 2 + ((colour + y + z0) & 1)) * HALF + jb;
      pd = Vec3{q0[0], q0[kLPF], q0[2 * kLPF]};
    }
    release(z0 - 1);
  }
  for (int k = z0; ok && k < z1; k++) {
    ok = wait_plane(k + 1);
    if (!ok) break;
    if (tid == 0 && !issue(k + kLNS - 1)) pfail = true;
    const int h = (colour + y + k) & 1;
    const int x = 2 * j + h;
    const bool valid = live_row && x < nx;
    const float *cs_k = slot_ptr(k);
    const float *above = plane_exists(k + 1) ? slot_ptr(k + 1) : nullptr;
    const float *own = cs_k + ((r + 1) * 2 + h) * HALF + jb;
    const float *oth = cs_k + ((r + 1) * 2 + (h ^ 1)) * HALF + jb - 1 + h;  // cells of x - 1, x + 1
    auto ld3 = [&](const float *p) { return Vec3{p[0], p[kLPF], p[2 * kLPF]}; };
    const Vec3 n = ld3(own);
    const Vec3 xm = ld3(oth), xp = ld3(oth + 1);
    Vec3 nb[6] = {xp, xm, ld3(own + RW), ld3(own - RW), above ? ld3(above + ((r + 1) * 2 + h) * HALF + jb)
                                                              : Vec3{0.f, 0.f, 0.f}, pd};
    float w[6];
    w[0] = (perx || x + 1 < nx) ? 1.f : 0.f;
    w[1] = (perx || x - 1 >= 0) ? 1.f : 0.f;
    w[2] = (pery || y + 1 < ny) ? 1.f : 0.f;
    w[3] = (pery || y - 1 >= 0) ? 1.f : 0.f;
    w[4] = above ? 1.f : 0.f;
    w[5] = plane_exists(k - 1) ? 1.f : 0.f;
#pragma unroll
    for (int d = 0; d < 6; d++)  // an absent neighbour is the zero vector, as the gathering kernel has it
      if (w[d] == 0.f) nb[d] = Vec3{0.f, 0.f, 0.f};
    pd = h ? xm : xp;  // the other-parity cell jb of plane k: the next step's -z neighbour
    release(k);         // plane k is not read again (plane k + 1, read above, is released at the next step)
    float f[kIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (valid) site_features(nb, w, St.T, f);
    float o[kOut];
    if (!wg_mlp_tc(T, &s_mma[wg], wfail, phase, a.timeout_ns, f, o)) break;  // warpgroup-uniform
    if (!valid) continue;
    int sid = -1;
    float sz = 0.f;
    if (GEO == GEO_SLAB) sid = slab_surface(k, nz, sz);
    const Vec3 sn{0.f, 0.f, sz};
    const Head hd = mlp_head(o, a.kappa_max);
    const U4 u = site_draws(R.seed, sweep, (uint32_t)site_linear(R, x, y, k), 1);
    const float em1 = expm1f(-2.f * hd.kappa), e2k = expf(-2.f * hd.kappa);
    const Vec3 nn = sample_proposal(hd, em1, e2k, u24(u.x), u24(u.y), u24(u.z), (u.x & 1u) != 0u);
    float b_old, b_new;
    bond_sum2<POT, false, true, float>(m, n, nn, nb, w, b_old, b_new);
    const float s_old = single_energy<true>(m, n, sid, sn, St.elecE);
    const float s_new = single_energy<true>(m, nn, sid, sn, St.elecE);
    const float dE = __fadd_rn(__fadd_rn(b_new, s_new), -__fadd_rn(b_old, s_old));
    bool acc;
    if (St.T > 0.f) {  // u < e^{-dE/T} q(n) / q(n'), without logarithms
      const float inv_den = -1.f / em1;
      const float q_old = q4pi(dot(hd.mu, n), hd.kappa, inv_den, e2k), q_new = q4pi(dot(hd.mu, nn), hd.kappa, inv_den, e2k);
      acc = u24(u.w) * q_new < __expf(-dE / St.T) * q_old;
    } else {
      acc = dE <= 0.f;
    }
    if (acc) {
      float *row0 = a.dir + R.off + ((long long)k * R.py + (y + GY)) * R.px + h * R.hp + GH;
      row0[j] = nn.x;
      row0[cs + j] = nn.y;
      row0[2 * cs + j] = nn.z;
      if ((perx && (j == 0 || j == (nx >> 1) - 1)) || (pery && (y < 2 || y >= ny - 2)))
        learned_ghosts(row0, cs, R.px, nn.x, nn.y, nn.z, j, nx, ny, y, perx, pery);
      accepted++;
    }
    if (measure) {  // the site is final: colour 0 adds its single-site terms, colour 1 2 bond + single
      const Vec3 nf = acc ? nn : n;
      const float bf = acc ? b_new : b_old, sf = acc ? s_new : s_old;
      dacc[0] += (double)(colour == 0 ? sf : __fadd_rn(__fmul_rn(2.f, bf), sf));
      dacc[1] += (double)fmaf(1.5f * nf.x, nf.x, -0.5f);
      dacc[2] += (double)(1.5f * nf.x * nf.y);
      dacc[3] += (double)(1.5f * nf.x * nf.z);
      dacc[4] += (double)fmaf(1.5f * nf.y, nf.y, -0.5f);
      dacc[5] += (double)(1.5f * nf.y * nf.z);
      dacc[6] += (double)fmaf(1.5f * nf.z, nf.z, -0.5f);
      dacc[7] += (double)nf.x;
      dacc[8] += (double)nf.y;
      dacc[9] += (double)nf.z;
    }
  }
  __syncthreads();  // both warpgroups have left the plane loop
  const int fl = s_wfail[0] | s_wfail[1];
  if (fl) {
    if (tid == 0) {
      atomicOr(a.err, (fl & 2) ? 2u : 1u);
      for (int q = max(waited + 1, last_issued - kLNS + 1); q <= last_issued; q++) {
        if (!plane_exists(q)) continue;
        const int lp = q - pbeg;
        mbar_wait_bounded(&bars[(unsigned)lp % kLNS], ((unsigned)lp / kLNS) & 1u, a.timeout_ns);
      }
    }
    tc_teardown(T);
    return;
  }
  const unsigned wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&a.st[it.rep].acc, (unsigned long long)wsum);
  if (measure) {
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < kPartials; q++) {
      double v = dacc[q];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (tid < kPartials) {
      double v = 0.0;
      for (int w2 = 0; w2 < kThreads / 32; w2++) v += red[w2][tid];
      double *dst = a.partials + (long long)blockIdx.x * kPartials + tid;
      *dst = colour == 0 ? v : *dst + v;
    }
  }
  tc_teardown(T);
}

template <int POT>
static cudaError_t learned_pass_pot(const ModelDev &m, const LearnedPassArgs &a, int geo, int n_items,
                                    cudaStream_t stream) {
  auto k = geo == GEO_SLAB ? k_learned_pass<POT, GEO_SLAB> : k_learned_pass<POT, GEO_BULK>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLearnedPassSmem);
  if (e != cudaSuccess) return e;
  k<<<n_items, kThreads, kLearnedPassSmem, stream>>>(m, a);
  return cudaGetLastError();
}

cudaError_t launch_learned_pass(const LaunchCtx &c, int geo, const LearnedPassView &v, const LearnedMlp &mlp,
                                float kappa_max, int measure, float *dir, int cur) {
  if (v.n_items == 0) return cudaSuccess;
  for (int colour = 0; colour < 2; colour++) {
    LearnedPassArgs a;
    a.tmaps = v.tmaps;
    a.dir = dir;
    a.reps = c.reps;
    a.st = c.state;
    a.items = v.items;
    a.partials = v.partials;
    a.sweep_ctr = c.sweep_ctr;
    a.mlp_tc = mlp.tc;
    a.err = mlp.err;
    a.kappa_max = kappa_max;
    a.cur = cur;
    a.colour = colour;
    a.measure = measure;
    a.timeout_ns = 2000000000ll;
    cudaError_t e;
    if (c.model.potential == POT_GHRL)
      e = learned_pass_pot<POT_GHRL>(c.model, a, geo, v.n_items, c.stream);
    else if (c.model.potential == POT_PEAR)
      e = learned_pass_pot<POT_PEAR>(c.model, a, geo, v.n_items, c.stream);
    else
      e = learned_pass_pot<POT_LL>(c.model, a, geo, v.n_items, c.stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// ---- launchers -------------------------------------------------------------------------------------------------
template <int POT, int GEO, bool TC>
static void sweep_learned_one(const LaunchCtx &c, const BlockTable &t, int colour, const LearnedMlp &mlp,
                              float kappa_max, int grid, int measure, double *partials) {
  auto k = k_sweep_learned<POT, GEO, TC>;
  const size_t smem = TC ? kTcMlpSmem : kWarpMlpSmem;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k<<<grid, kThreads, smem, c.stream>>>(c.model, c.reps, c.state, c.dir, c.pt, c.nrm, c.sweep_ctr, colour, t.rep,
                                        t.base, t.n_blocks, mlp.warp, mlp.tc, mlp.err, kappa_max, measure, partials);
}

template <int POT>
static void sweep_learned_pot(const LaunchCtx &c, int geo, const BlockTable &t, int colour, const LearnedMlp &mlp,
                              float kappa_max, int grid, int measure, double *partials) {
  if (mlp.use_tc) {
    if (geo == GEO_BULK)
      sweep_learned_one<POT, GEO_BULK, true>(c, t, colour, mlp, kappa_max, grid, measure, partials);
    else if (geo == GEO_SLAB)
      sweep_learned_one<POT, GEO_SLAB, true>(c, t, colour, mlp, kappa_max, grid, measure, partials);
    else
      sweep_learned_one<POT, GEO_PT, true>(c, t, colour, mlp, kappa_max, grid, measure, partials);
    return;
  }
  if (geo == GEO_BULK)
    sweep_learned_one<POT, GEO_BULK, false>(c, t, colour, mlp, kappa_max, grid, measure, partials);
  else if (geo == GEO_SLAB)
    sweep_learned_one<POT, GEO_SLAB, false>(c, t, colour, mlp, kappa_max, grid, measure, partials);
  else
    sweep_learned_one<POT, GEO_PT, false>(c, t, colour, mlp, kappa_max, grid, measure, partials);
}

cudaError_t launch_sweep_learned(const LaunchCtx &c, int geo, const BlockTable &half, const LearnedMlp &mlp,
                                 float kappa_max, int measure, double *partials) {
  if (half.n_blocks == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::min(half.n_blocks, sms * 8);
  for (int colour = 0; colour < 2; colour++) {
    if (c.model.potential == POT_GHRL)
      sweep_learned_pot<POT_GHRL>(c, geo, half, colour, mlp, kappa_max, grid, measure, partials);
    else if (c.model.potential == POT_PEAR)
      sweep_learned_pot<POT_PEAR>(c, geo, half, colour, mlp, kappa_max, grid, measure, partials);
    else
      sweep_learned_pot<POT_LL>(c, geo, half, colour, mlp, kappa_max, grid, measure, partials);
  }
  return cudaGetLastError();
}

}  // namespace mcl

// ---- C ABI -----------------------------------------------------------------------------------------------------
using namespace mcl;

#define CKL(call)                                        \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

struct mcl_trainer {
  long long max_batch = 0;
  int max_blocks = 0;
  float kappa_max = 500.f;
  float *d_params = nullptr, *d_wr = nullptr, *d_m1 = nullptr, *d_m2 = nullptr, *d_partial = nullptr;
  double *d_grad = nullptr;
  long long steps = 0;
  cudaStream_t stream = nullptr;
};

static bool finite_params(const mcl_mlp *p) {
  const float *f = reinterpret_cast<const float *>(p);
  for (int i = 0; i < kNP; i++)
    if (!std::isfinite(f[i])) return false;
  return true;
}

namespace mcl {
int learned_check_error(mcl_engine *e) {
  if (!e->d_lerr) return MCL_OK;
  unsigned v = 0;
  CKL(cudaMemcpyAsync(&v, e->d_lerr, sizeof v, cudaMemcpyDeviceToHost, e->stream));
  CKL(cudaStreamSynchronize(e->stream));
  return learned_report_error(e, v);
}

int learned_report_error(mcl_engine *e, unsigned v) {
  if (!v || !e->d_lerr) return MCL_OK;
  CKL(cudaMemsetAsync(e->d_lerr, 0, sizeof v, e->stream));
  return fail(MCL_ERR_CUDA, (v & 2u) ? "learned sweep: a plane copy did not arrive within 2 s"
                                     : "learned sweep: a tensor-core completion did not arrive within 2 s");
}
}  // namespace mcl

extern "C" {

int mcl_set_proposal(mcl_engine *e, const mcl_mlp *mlp, float kappa_max) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (mlp && e->zslab) return fail(MCL_ERR_STATE, "mcl_set_proposal: a z-slab engine runs the plain proposal only");
  CKL(cudaStreamSynchronize(e->stream));
  if (!mlp) {
    if (e->d_mlp) cudaFree(e->d_mlp);
    e->d_mlp = nullptr;
    return MCL_OK;
  }
  if (!(kappa_max > kKappaMin && kappa_max <= 1e4f))
    return fail(MCL_ERR_ARG, "mcl_set_proposal: kappa_max must lie in (1e-3, 1e4]");
  if (!finite_params(mlp)) return fail(MCL_ERR_NONFINITE, "mcl_set_proposal: non-finite weight");
  MlpDev h;
  to_device_layout(*mlp, h);
  MlpTC ht;
  to_tc_layout(*mlp, ht);
  if (!e->d_mlp) CKL(cudaMalloc(&e->d_mlp, sizeof(MlpDev)));
  if (!e->d_mlp_tc) CKL(cudaMalloc(&e->d_mlp_tc, sizeof(MlpTC)));
  if (!e->d_lerr) {
    CKL(cudaMalloc(&e->d_lerr, sizeof(unsigned)));
    CKL(cudaMemset(e->d_lerr, 0, sizeof(unsigned)));
  }
  CKL(cudaMemcpy(e->d_mlp, &h, sizeof h, cudaMemcpyHostToDevice));
  CKL(cudaMemcpy(e->d_mlp_tc, &ht, sizeof ht, cudaMemcpyHostToDevice));
  e->kappa_max = kappa_max;
  // tcgen05 unless MCL_LEARNED_MLP=mma selects the mma.sync warps (same network, same rounding points)
  const char *path = getenv("MCL_LEARNED_MLP");
  e->mlp_tc = !(path && strcmp(path, "mma") == 0);
  // colour passes on streamed planes where the engine tiles (bulk, slab), unless MCL_LEARNED_KERNEL=gather
  // selects the kernel that gathers each site's neighbours from global memory (same decisions)
  const char *kern = getenv("MCL_LEARNED_KERNEL");
  e->learned_pass = !(kern && strcmp(kern, "gather") == 0);
  return MCL_OK;
}

int mcl_extract_samples(mcl_engine *e, int replica, long long n, unsigned long long seed, float *d_features,
                        float *d_directors) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (replica < 0 || replica >= e->n_rep) return fail(MCL_ERR_ARG, "replica %d outside 0..%d", replica, e->n_rep - 1);
  if (n < 0 || (n > 0 && (!d_features || !d_directors))) return fail(MCL_ERR_ARG, "mcl_extract_samples: bad buffers");
  if (!e->geometry_set) return fail(MCL_ERR_STATE, "custom geometry: call mcl_set_geometry first");
  if (n == 0) return MCL_OK;
  const LaunchCtx c = e->ctx();
  const int threads = 256;
  const long long blocks = (n + threads - 1) / threads;
  if (blocks > 0x7FFFFFFFll) return fail(MCL_ERR_ARG, "mcl_extract_samples: too many samples");
  switch (e->geo) {
    case GEO_BULK:
      k_extract_samples<GEO_BULK><<<(unsigned)blocks, threads, 0, c.stream>>>(c.reps, c.state, c.dir, c.pt, c.nrm,
                                                                              replica, n, seed, d_features, d_directors);
      break;
    case GEO_SLAB:
      k_extract_samples<GEO_SLAB><<<(unsigned)blocks, threads, 0, c.stream>>>(c.reps, c.state, c.dir, c.pt, c.nrm,
                                                                              replica, n, seed, d_features, d_directors);
      break;
    default:
      k_extract_samples<GEO_PT><<<(unsigned)blocks, threads, 0, c.stream>>>(c.reps, c.state, c.dir, c.pt, c.nrm,
                                                                            replica, n, seed, d_features, d_directors);
  }
  CKL(cudaGetLastError());
  e->launches++;
  CKL(cudaStreamSynchronize(c.stream));
  return MCL_OK;
}

int mcl_mlp_forward(const mcl_mlp *mlp, const float *d_features, long long n, float *d_out, void *stream) {
  if (!mlp || n < 0 || (n > 0 && (!d_features || !d_out))) return fail(MCL_ERR_ARG, "mcl_mlp_forward: bad arguments");
  if (n == 0) return MCL_OK;
  MlpDev h;
  to_device_layout(*mlp, h);
  MlpDev *d = nullptr;
  CKL(cudaMalloc(&d, sizeof h));
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t err = cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) {
    const long long blocks = std::min<long long>((n + kThreads - 1) / kThreads, 148ll * 16);
    k_mlp_forward<<<(unsigned)blocks, kThreads, 0, st>>>(d, d_features, n, d_out);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  cudaFree(d);
  if (err != cudaSuccess) return cuda_fail(err, "mcl_mlp_forward");
  return MCL_OK;
}

int mcl_mlp_forward_tcgen05(const mcl_mlp *mlp, const float *d_features, long long n, float *d_out, void *stream) {
  if (!mlp || n < 0 || (n > 0 && (!d_features || !d_out)))
    return fail(MCL_ERR_ARG, "mcl_mlp_forward_tcgen05: bad arguments");
  if (n == 0) return MCL_OK;
  MlpTC h;
  to_tc_layout(*mlp, h);
  MlpTC *d = nullptr;
  unsigned *err = nullptr;
  CKL(cudaMalloc(&d, sizeof h));
  cudaError_t e2 = cudaMalloc(&err, sizeof(unsigned));
  if (e2 != cudaSuccess) {
    cudaFree(d);
    return cuda_fail(e2, "cudaMalloc");
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = sizeof(TcSmem) + 128;
  cudaError_t e = cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(unsigned), st);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    const long long blocks = std::min<long long>((n + kTcRows - 1) / kTcRows, 148ll * 2);
    k_mlp_forward_tc<<<(unsigned)blocks, kTcRows, smem, st>>>(d, d_features, n, d_out, err, 2000000000ll);
    e = cudaGetLastError();
  }
  unsigned flag = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof flag, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d);
  cudaFree(err);
  if (e != cudaSuccess) return cuda_fail(e, "mcl_mlp_forward_tcgen05");
  if (flag) return fail(MCL_ERR_CUDA, "mcl_mlp_forward_tcgen05: a tensor-core commit did not arrive in time");
  return MCL_OK;
}

int mcl_trainer_create(const mcl_mlp *init, long long max_batch, float kappa_max, mcl_trainer **out) {
  if (!init || !out || max_batch < 1) return fail(MCL_ERR_ARG, "mcl_trainer_create: bad arguments");
  *out = nullptr;
  if (!(kappa_max > kKappaMin && kappa_max <= 1e4f)) return fail(MCL_ERR_ARG, "mcl_trainer_create: bad kappa_max");
  if (!finite_params(init)) return fail(MCL_ERR_NONFINITE, "mcl_trainer_create: non-finite weight");
  const long long nb = (max_batch + kTB - 1) / kTB;
  if (nb > (1 << 24)) return fail(MCL_ERR_ARG, "mcl_trainer_create: max_batch too large");
  mcl_trainer *t = new mcl_trainer();
  t->max_batch = max_batch;
  t->max_blocks = (int)nb;
  t->kappa_max = kappa_max;
  auto bad = [&](cudaError_t err, const char *what) {
    mcl_trainer_destroy(t);
    return cuda_fail(err, what);
  };
  cudaError_t err;
  if ((err = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking)) != cudaSuccess) return bad(err, "stream");
  if ((err = cudaMalloc(&t->d_params, kNP * sizeof(float))) != cudaSuccess) return bad(err, "cudaMalloc");
  if ((err = cudaMalloc(&t->d_wr, kNP * sizeof(float))) != cudaSuccess) return bad(err, "cudaMalloc");
  if ((err = cudaMalloc(&t->d_m1, kNP * sizeof(float))) != cudaSuccess) return bad(err, "cudaMalloc");
  if ((err = cudaMalloc(&t->d_m2, kNP * sizeof(float))) != cudaSuccess) return bad(err, "cudaMalloc");
  if ((err = cudaMalloc(&t->d_grad, (kNP + 1) * sizeof(double))) != cudaSuccess) return bad(err, "cudaMalloc");
  if ((err = cudaMalloc(&t->d_partial, (size_t)nb * (kNP + 1) * sizeof(float))) != cudaSuccess)
    return bad(err, "cudaMalloc");
  if ((err = cudaMemcpy(t->d_params, init, kNP * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
    return bad(err, "cudaMemcpy");
  if ((err = cudaMemset(t->d_m1, 0, kNP * sizeof(float))) != cudaSuccess) return bad(err, "cudaMemset");
  if ((err = cudaMemset(t->d_m2, 0, kNP * sizeof(float))) != cudaSuccess) return bad(err, "cudaMemset");
  k_round<<<(kNP + 255) / 256, 256, 0, t->stream>>>(t->d_params, t->d_wr);
  if ((err = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem)) !=
      cudaSuccess)
    return bad(err, "cudaFuncSetAttribute");
  if ((err = cudaStreamSynchronize(t->stream)) != cudaSuccess) return bad(err, "k_round");
  *out = t;
  return MCL_OK;
}

static int trainer_grad(mcl_trainer *t, const float *d_features, const float *d_directors, long long n) {
  if (!t || !d_features || !d_directors || n < 1) return fail(MCL_ERR_ARG, "trainer: bad arguments");
  if (n > t->max_batch) return fail(MCL_ERR_ARG, "trainer: batch %lld exceeds max_batch %lld", n, t->max_batch);
  const int nb = (int)((n + kTB - 1) / kTB);
  k_mlp_grad<<<nb, kTB, kTrainSmem, t->stream>>>(t->d_wr, d_features, d_directors, n, t->kappa_max, 1.f / (float)n,
                                                t->d_partial);
  CKL(cudaGetLastError());
  k_grad_reduce<<<(kNP + 1 + 255) / 256, 256, 0, t->stream>>>(t->d_partial, nb, t->d_grad);
  CKL(cudaGetLastError());
  return MCL_OK;
}

int mcl_trainer_gradient(mcl_trainer *t, const float *d_features, const float *d_directors, long long n,
                         mcl_mlp *grad, double *loss) {
  int rc = trainer_grad(t, d_features, d_directors, n);
  if (rc) return rc;
  std::vector<double> g(kNP + 1);
  CKL(cudaMemcpyAsync(g.data(), t->d_grad, (kNP + 1) * sizeof(double), cudaMemcpyDeviceToHost, t->stream));
  CKL(cudaStreamSynchronize(t->stream));
  if (grad) {
    float *f = reinterpret_cast<float *>(grad);
    for (int i = 0; i < kNP; i++) f[i] = (float)g[i];
  }
  if (loss) *loss = g[kNP] / (double)n;
  return MCL_OK;
}

int mcl_trainer_step(mcl_trainer *t, const float *d_features, const float *d_directors, long long n, float lr,
                     double *loss) {
  if (!(lr > 0.f && lr < 1.f)) return fail(MCL_ERR_ARG, "mcl_trainer_step: learning rate must lie in (0, 1)");
  int rc = trainer_grad(t, d_features, d_directors, n);
  if (rc) return rc;
  t->steps++;
  const float bc1 = 1.f - powf(0.9f, (float)t->steps), bc2 = 1.f - powf(0.999f, (float)t->steps);
  k_adam<<<(kNP + 255) / 256, 256, 0, t->stream>>>(t->d_grad, t->d_params, t->d_wr, t->d_m1, t->d_m2, lr, bc1, bc2);
  CKL(cudaGetLastError());
  if (loss) {
    double l = 0.0;
    CKL(cudaMemcpyAsync(&l, t->d_grad + kNP, sizeof(double), cudaMemcpyDeviceToHost, t->stream));
    CKL(cudaStreamSynchronize(t->stream));
    *loss = l / (double)n;
  }
  return MCL_OK;
}

int mcl_trainer_get(mcl_trainer *t, mcl_mlp *out) {
  if (!t || !out) return fail(MCL_ERR_ARG, "mcl_trainer_get: null argument");
  CKL(cudaStreamSynchronize(t->stream));
  CKL(cudaMemcpy(out, t->d_params, kNP * sizeof(float), cudaMemcpyDeviceToHost));
  return MCL_OK;
}

int mcl_trainer_destroy(mcl_trainer *t) {
  if (!t) return MCL_OK;
  if (t->stream) cudaStreamSynchronize(t->stream);
  cudaFree(t->d_params);
  cudaFree(t->d_wr);
  cudaFree(t->d_m1);
  cudaFree(t->d_m2);
  cudaFree(t->d_grad);
  cudaFree(t->d_partial);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return MCL_OK;
}

}  // extern "C"
