// The proposal MLP on Blackwell's fifth-generation tensor cores (tcgen05): one CTA of 256 threads evaluates 256
// rows (sites) as two 128-row tiles. Operands sit in shared memory in the no-swizzle K-major core-matrix layout
// (8 rows x 16 bytes per core matrix; core matrices adjacent along K are 128 bytes apart, along M/N (K/8) x 128
// bytes), accumulators in tensor memory (64 FP32 columns per tile, lane = row). One thread issues
// tcgen05.mma (M = 128, N = 64 or 16, K = 16 per instruction, BF16 x BF16 -> FP32) and commits to an mbarrier;
// every thread then reads its own row back with tcgen05.ld (warp w reads lanes 32 (w % 4) .. of tile w / 4),
// applies bias and SiLU in registers, and writes the BF16 row of the next layer's A operand.
//
// Weights and biases of the two hidden layers are stored halved (exact), so that the accumulators hold h = z / 2
// and SiLU is h + h tanh(h), as in the mma.sync path; the BF16 rounding points are the same.
//
// Every mbarrier wait is bounded by %globaltimer: on timeout the CTA records an error, waits (bounded) for the
// commit in flight, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mcl {

// Weights in the core-matrix layout (global memory; copied to shared memory per CTA).
struct MlpTC {
  uint8_t w1[2048];   // N = 64 x K = 16 (K 7..15 zero)
  uint8_t w2[8192];   // N = 64 x K = 64
  uint8_t w3[2048];   // N = 16 (rows 4..15 zero) x K = 64
  float b1[64], b2[64], b3[16];
};
static_assert(sizeof(MlpTC) % 16 == 0, "MlpTC is copied in 16-byte words");

// Byte offset of element (row r, column k) in a K-major core-matrix tile with kt columns.
__host__ __device__ constexpr int core_off(int r, int k, int kt) {
  return ((r >> 3) * (kt >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

constexpr int kTcRows = 256;                 // rows (sites) per CTA pass
constexpr int kTcA1 = 128 * 16 * 2;          // one 128-row tile of layer-1 input (K = 16), bytes
constexpr int kTcA2 = 128 * 64 * 2;          // one 128-row tile of a hidden layer (K = 64), bytes
constexpr int kTcCols = 128;                 // tensor-memory columns per CTA (2 tiles x 64)

struct TcSmem {
  alignas(128) uint8_t w1[2048];
  alignas(128) uint8_t w2[8192];
  alignas(128) uint8_t w3[2048];
  alignas(128) uint8_t a1[2 * kTcA1];
  alignas(128) uint8_t a2[2 * kTcA2];
  float b1[64], b2[64], b3[16];
  unsigned long long bar;
  uint32_t tmem;
  int fail;
};

__device__ __forceinline__ uint32_t tc_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// A dynamic shared-memory array rounded up to 128 bytes by an offset from the array itself, so that accesses
// through the result stay in the shared address space.
__device__ __forceinline__ unsigned char *tc_align128(unsigned char *base) {
  return base + ((128u - (tc_smem(base) & 127u)) & 127u);
}

__device__ __forceinline__ uint64_t tc_desc(const void *start, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((tc_smem(start) & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
         ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t tc_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_ld4(uint32_t taddr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 4; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ bool tc_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(tc_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint: a thread whose phase is not complete sleeps (up to hint_ns) instead of
// returning at once, so the threads waiting for an MMA stage take no issue slots from the SM's other CTAs.
__device__ __forceinline__ bool tc_try_wait_sleep(unsigned long long *bar, unsigned parity, unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(tc_smem(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool tc_wait(unsigned long long *bar, unsigned parity, long long timeout_ns) {
  if (tc_try_wait(bar, parity)) return true;
  unsigned long long t0;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t0));
  while (true) {
    if (tc_try_wait_sleep(bar, parity, 20000u)) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    if ((long long)(t - t0) > timeout_ns) return false;
  }
}

// Set-up of a CTA of 256 threads: weights to shared memory, mbarrier, 128 tensor-memory columns (warp 0).
__device__ __forceinline__ void tc_setup(TcSmem &S, const MlpTC *__restrict__ w) {
  const int tid = threadIdx.x;
  const uint4 *src = reinterpret_cast<const uint4 *>(w);
  for (int i = tid; i < (int)(sizeof(w->w1) / 16); i += blockDim.x)
    reinterpret_cast<uint4 *>(S.w1)[i] = src[i];
  for (int i = tid; i < (int)(sizeof(w->w2) / 16); i += blockDim.x)
    reinterpret_cast<uint4 *>(S.w2)[i] = src[sizeof(w->w1) / 16 + i];
  for (int i = tid; i < (int)(sizeof(w->w3) / 16); i += blockDim.x)
    reinterpret_cast<uint4 *>(S.w3)[i] = src[(sizeof(w->w1) + sizeof(w->w2)) / 16 + i];
  for (int i = tid; i < 64; i += blockDim.x) {
    S.b1[i] = w->b1[i];
    S.b2[i] = w->b2[i];
  }
  if (tid < 16) S.b3[tid] = w->b3[tid];
  if (tid == 0) {
    S.fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&S.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&S.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// Frees the tensor memory (all threads call it; warp 0 deallocates after every thread's loads are done).
__device__ __forceinline__ void tc_teardown(TcSmem &S) {
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(kTcCols) : "memory");
  }
}

// One MMA stage: thread 0 issues the stage's instructions for both tiles and commits; every thread waits. Returns
// false (CTA-uniform) if the commit did not arrive within the time limit.
template <typename Issue>
__device__ __forceinline__ bool tc_stage(TcSmem &S, unsigned &phase, long long timeout_ns, Issue issue) {
  tc_fence_async_smem();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    issue();
    tc_commit(&S.bar);
  }
  const bool ok = tc_wait(&S.bar, phase, timeout_ns);
  if (!ok) atomicExch(&S.fail, 1);
  __syncthreads();
  const bool cta_ok = S.fail == 0;
  if (!cta_ok) {  // wait (bounded) for the commit in flight before anybody frees the tensor memory
    tc_wait(&S.bar, phase, timeout_ns);
    return false;
  }
  phase ^= 1u;
  tc_fence_after();
  return true;
}

}  // namespace mcl
