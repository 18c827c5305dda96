// mcl_observe_device: the observables of a director field that already lives in device memory, computed without
// allocating anything. It is the observation kernel of the engine (kernels.cu k_observe + k_finalize) recast for
// callers that hold their own director buffer and may not allocate device memory at the moment they measure,
// e.g. a host that has handed all of the device's memory to its own pool allocator, or a timing loop in which an
// implicit device-wide synchronisation from cudaMalloc/cudaFree is not acceptable.
//
// The per-block partial sums and the final record go to one file-scope __device__ array instead of engine
// buffers. Its size fixes the largest lattice this entry point takes (kStaticSlots blocks of kSitesPerSlot sites,
// 2^26 sites); larger requests are rejected with MCL_ERR_ARG. The array's address is looked up once per device by
// the first call on that device. Since there is one array per device, calls on the same device must not overlap.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "eigen3.cuh"
#include "engine.h"
#include "physics.cuh"
#include "site_access.cuh"

namespace mcl {
namespace {

constexpr int kSitesPerSlot = 4096;                      // sites one block sums into one partial slot
constexpr int kStaticSlots = 16384;                      // partial slots in the scratch array
constexpr long long kStaticMaxSites = (long long)kStaticSlots * kSitesPerSlot;  // 2^26
constexpr int kRecordDoubles = (int)(sizeof(ObsRecord) / sizeof(double));
constexpr long long kRecordOffset = (long long)kStaticSlots * kPartials;       // in doubles; 256-byte aligned
constexpr int kMaxDevices = 64;

static_assert(sizeof(ObsRecord) == sizeof(mcl_observables), "ObsRecord must match mcl_observables");
static_assert((kRecordOffset * sizeof(double)) % 256 == 0, "record offset alignment");

#define CK_STATIC(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Scratch of mcl_observe_device, 1.25 MiB per device: kStaticSlots x kPartials partial sums, then one ObsRecord.
// Every block writes all kPartials values of its own slot before the finalisation kernel reads them, and the
// record is written whole by that kernel, so no part of it has to start at zero or be cleared between calls.
static __device__ __align__(256) double g_observe_scratch[kRecordOffset + kRecordDoubles];

// Unpadded lattice of the caller's buffer: 3 floats per site, site (x, y, z) at x + nx (y + ny z).
struct PlainLattice {
  int nx, ny, nz;
  int periodic[3];
  long long n_sites;
};

__device__ __forceinline__ double warp_sum_static(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ Vec3 load_plain(const float *__restrict__ ni, long long site) {
  return Vec3{__ldg(ni + 3 * site), __ldg(ni + 3 * site + 1), __ldg(ni + 3 * site + 2)};
}

// Block b sums sites [b kSitesPerSlot, (b + 1) kSitesPerSlot) into slot b: site energy (bonds with the same
// neighbour rules as the engine, anchoring on the slab surfaces, field), (3 n n - I)/2 and n, in FP64.
template <int POT, int GEO>
__global__ void __launch_bounds__(kThreads) k_observe_static(ModelDev m, PlainLattice L, float elecE,
                                                             const float *__restrict__ ni,
                                                             double *__restrict__ partials) {
  const long long base = (long long)blockIdx.x * kSitesPerSlot;
  const long long end = min(base + (long long)kSitesPerSlot, L.n_sites);
  double acc[kPartials];
#pragma unroll
  for (int k = 0; k < kPartials; k++) acc[k] = 0.0;
  for (long long q = base + threadIdx.x; q < end; q += kThreads) {
    const int x = (int)(q % L.nx);
    const long long row = q / L.nx;
    const int y = (int)(row % L.ny), z = (int)(row / L.ny);
    const Vec3 n = load_plain(ni, q);
    Vec3 nb[6];
    float w[6];
#pragma unroll
    for (int d = 0; d < 6; d++) {
      const int axis = d >> 1;
      const int delta = (d & 1) ? -1 : 1;
      int xx = x, yy = y, zz = z;
      bool ok;
      if (axis == 0)
        ok = nb_coord(L.periodic[0], x + delta, L.nx, xx);
      else if (axis == 1)
        ok = nb_coord(L.periodic[1], y + delta, L.ny, yy);
      else
        ok = nb_coord(L.periodic[2], z + delta, L.nz, zz);
      if (ok) {
        nb[d] = load_plain(ni, (long long)xx + (long long)L.nx * ((long long)yy + (long long)L.ny * zz));
        w[d] = 1.f;
      } else {
        nb[d] = Vec3{0.f, 0.f, 0.f};
        w[d] = 0.f;
      }
    }
    int sid = -1;
    Vec3 s{0.f, 0.f, 0.f};
    if (GEO == GEO_SLAB) {
      float sz;
      sid = slab_surface(z, L.nz, sz);
      s.z = sz;
    }
    acc[0] += (double)site_energy<POT>(m, n, nb, w, sid, s, elecE);
    const double nx = n.x, ny = n.y, nz = n.z;
    acc[1] += 1.5 * nx * nx - 0.5;
    acc[2] += 1.5 * nx * ny;
    acc[3] += 1.5 * nx * nz;
    acc[4] += 1.5 * ny * ny - 0.5;
    acc[5] += 1.5 * ny * nz;
    acc[6] += 1.5 * nz * nz - 0.5;
    acc[7] += nx;
    acc[8] += ny;
    acc[9] += nz;
  }
  __shared__ double red[kThreads / 32][kPartials];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kPartials; k++) {
    const double v = warp_sum_static(acc[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kPartials) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; w++) v += red[w][threadIdx.x];
    partials[(long long)blockIdx.x * kPartials + threadIdx.x] = v;
  }
}

// One block: fixed-order reduction of the n_slots partial slots, then S and the director (Jacobi, eigen3.cuh).
__global__ void __launch_bounds__(kThreads) k_observe_static_finalize(int n_slots, double n_valid, double ang_var,
                                                                      const double *__restrict__ partials,
                                                                      ObsRecord *__restrict__ out) {
  __shared__ double red[kThreads / 32][kPartials];
  __shared__ double tot[kPartials];
  double acc[kPartials];
#pragma unroll
  for (int k = 0; k < kPartials; k++) acc[k] = 0.0;
  for (int b = threadIdx.x; b < n_slots; b += kThreads)
#pragma unroll
    for (int k = 0; k < kPartials; k++) acc[k] += partials[(long long)b * kPartials + k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kPartials; k++) {
    const double v = warp_sum_static(acc[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kPartials) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; w++) v += red[w][threadIdx.x];
    tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ObsRecord o;
    o.energy = tot[0] / n_valid;
    for (int k = 0; k < 6; k++) o.q[k] = tot[1 + k] / n_valid;
    double vec[3];
    o.S = largest_eigen3(o.q, vec);
    for (int k = 0; k < 3; k++) {
      o.director[k] = vec[k];
      o.nsum[k] = tot[7 + k];
    }
    o.n_valid = n_valid;
    o.acceptance = 0.0;
    o.ang_var = ang_var;
    o.sweep = 0.0;
    *out = o;
  }
}

template <int POT>
void launch_observe_static(int geo, int n_slots, const ModelDev &m, const PlainLattice &L, float elecE,
                           const float *ni, double *partials, cudaStream_t stream) {
  if (geo == GEO_SLAB)
    k_observe_static<POT, GEO_SLAB><<<n_slots, kThreads, 0, stream>>>(m, L, elecE, ni, partials);
  else
    k_observe_static<POT, GEO_BULK><<<n_slots, kThreads, 0, stream>>>(m, L, elecE, ni, partials);
}

// Address of g_observe_scratch on each device, looked up by the first call made with that device current.
std::mutex g_scratch_mu;
double *g_scratch_addr[kMaxDevices] = {};

int scratch_address(int dev, double **out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_observe_scratch);
    if (err != cudaSuccess) return cuda_fail(err, "mcl_observe_device: cudaGetSymbolAddress of the scratch array");
    g_scratch_addr[dev] = (double *)p;
  }
  *out = g_scratch_addr[dev];
  return MCL_OK;
}

typedef CUresult (*AddressRangeFn)(CUdeviceptr *, size_t *, CUdeviceptr);

AddressRangeFn get_address_range() {
  static AddressRangeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (AddressRangeFn)p;
  });
  return fn;
}

typedef CUresult (*PointerAttributeFn)(void *, CUpointer_attribute, CUdeviceptr);

PointerAttributeFn get_pointer_attribute() {
  static PointerAttributeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PointerAttributeFn)p;
  });
  return fn;
}

// Whether ptr lies in memory mapped through the virtual-memory-management API (cuMemCreate + cuMemMap): such memory
// is not usable with the legacy IPC calls, memory from cudaMalloc is.
bool vmm_mapped(CUdeviceptr ptr) {
  PointerAttributeFn attr = get_pointer_attribute();
  int legacy = 1;
  return attr && attr(&legacy, CU_POINTER_ATTRIBUTE_IS_LEGACY_CUDA_IPC_CAPABLE, ptr) == CUDA_SUCCESS && legacy == 0;
}

// The caller's buffer must be memory of the current device (or managed memory) holding 3 n_sites floats.
int check_buffer(const float *d_ni, long long n_sites, int dev) {
  if (((uintptr_t)d_ni & 3u) != 0) return fail(MCL_ERR_ARG, "mcl_observe_device: d_ni is not 4-byte aligned");
  cudaPointerAttributes a;
  cudaError_t err = cudaPointerGetAttributes(&a, d_ni);
  if (err != cudaSuccess) {
    cudaGetLastError();
    return fail(MCL_ERR_ARG, "mcl_observe_device: d_ni is not a CUDA pointer (%s)", cudaGetErrorString(err));
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return fail(MCL_ERR_ARG, "mcl_observe_device: d_ni is not device memory (pointer type %d)", (int)a.type);
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    return fail(MCL_ERR_ARG, "mcl_observe_device: d_ni is memory of device %d but device %d is current", a.device,
                dev);
  AddressRangeFn range = get_address_range();
  CUdeviceptr lo = 0;
  size_t size = 0;
  if (!range || range(&lo, &size, (CUdeviceptr)(uintptr_t)d_ni) != CUDA_SUCCESS)
    return fail(MCL_ERR_ARG, "mcl_observe_device: cannot determine the allocation that holds d_ni");
  const unsigned long long need = (unsigned long long)n_sites * 3ull * sizeof(float);
  const unsigned long long start = (unsigned long long)(uintptr_t)d_ni;
  if (start < lo) return fail(MCL_ERR_ARG, "mcl_observe_device: d_ni lies outside the allocation reported for it");
  unsigned long long end = (unsigned long long)lo + size;
  if (end < start + need && !vmm_mapped((CUdeviceptr)start))
    return fail(MCL_ERR_ARG,
                "mcl_observe_device: d_ni must hold %llu bytes (3 floats per site) but its allocation ends %llu "
                "bytes after it",
                need, end - start);
  // Pool allocators built on virtual memory management (cuMemCreate + cuMemMap, e.g. torch's expandable segments)
  // map one buffer as several consecutive physical chunks, and the range query reports one chunk: such a buffer is
  // accepted when consecutive mapped ranges, each starting where the previous one ends, cover it.
  while (end < start + need) {
    CUdeviceptr lo2 = 0;
    size_t size2 = 0;
    if (range(&lo2, &size2, (CUdeviceptr)end) != CUDA_SUCCESS || (unsigned long long)lo2 != end || size2 == 0)
      return fail(MCL_ERR_ARG,
                  "mcl_observe_device: d_ni must hold %llu bytes (3 floats per site) but the mapped memory from it "
                  "ends %llu bytes after it",
                  need, end - start);
    end = (unsigned long long)lo2 + size2;
  }
  return MCL_OK;
}

// Lab easy axis of an anchoring from (theta, phi) in degrees, float host libm as in src/anchoring.cpp:19-24.
void easy_axis(float theta_deg, float phi_deg, float out[3]) {
  const float toRad = (float)(M_PI / 180);
  out[0] = sinf(toRad * theta_deg) * cosf(toRad * phi_deg);
  out[1] = sinf(toRad * theta_deg) * sinf(toRad * phi_deg);
  out[2] = cosf(toRad * theta_deg);
}

}  // namespace
}  // namespace mcl

using namespace mcl;

extern "C" int mcl_observe_device(const mcl_model *model, const mcl_replica *replica, const float *d_ni,
                                  mcl_observables *out, void *stream) {
  if (!model || !replica || !d_ni || !out) return fail(MCL_ERR_ARG, "mcl_observe_device: null argument");
  if (model->potential < MCL_POT_LL || model->potential > MCL_POT_PEAR)
    return fail(MCL_ERR_ARG, "mcl_observe_device: unknown potential %d", model->potential);
  if (model->n_surfaces < 0 || model->n_surfaces > MCL_MAX_SURFACES)
    return fail(MCL_ERR_ARG, "mcl_observe_device: n_surfaces %d outside 0..%d", model->n_surfaces, MCL_MAX_SURFACES);
  for (int s = 0; s < model->n_surfaces; s++)
    if (model->anch_type[s] < MCL_ANCH_HOMEOTROPIC || model->anch_type[s] > MCL_ANCH_FG_GHRL)
      return fail(MCL_ERR_ARG, "mcl_observe_device: unknown anchoring type %d of surface %d", model->anch_type[s], s);
  const mcl_replica &R = *replica;
  if (R.geometry != MCL_GEOM_BULK && R.geometry != MCL_GEOM_SLAB)
    return fail(MCL_ERR_ARG,
                "mcl_observe_device: geometry %d is not bulk or slab; sphere and custom lattices need the point-type "
                "tables of an engine (mcl_measure)",
                R.geometry);
  if (R.geometry == MCL_GEOM_SLAB && model->n_surfaces < 2)
    return fail(MCL_ERR_ARG, "mcl_observe_device: slab geometry needs anchoring for surfaces 0 and 1");
  if (R.nx < 1 || R.ny < 1 || R.nz < 1) return fail(MCL_ERR_ARG, "mcl_observe_device: grid sizes must be >= 1");
  const long long n_sites = (long long)R.nx * R.ny * R.nz;
  if (n_sites > kStaticMaxSites)
    return fail(MCL_ERR_ARG,
                "mcl_observe_device: %lld sites exceed the limit of %lld (its fixed scratch holds %d partial sums of "
                "%d sites); measure larger lattices through an engine (mcl_measure)",
                n_sites, kStaticMaxSites, kStaticSlots, kSitesPerSlot);

  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return fail(MCL_ERR_NO_DEVICE, "mcl_observe_device: no CUDA device: %s", cudaGetErrorString(ce));
  if (dev < 0 || dev >= kMaxDevices) return fail(MCL_ERR_ARG, "mcl_observe_device: device index %d >= %d", dev, kMaxDevices);
  int rc = check_buffer(d_ni, n_sites, dev);
  if (rc) return rc;
  double *scratch = nullptr;
  if ((rc = scratch_address(dev, &scratch))) return rc;

  ModelDev m;
  memset(&m, 0, sizeof m);
  m.potential = model->potential;
  m.A = model->A;
  m.B1 = model->B1;
  m.C = model->C;
  m.lam = model->ghrl_lambda;
  m.mu = model->ghrl_mu;
  m.nu = model->ghrl_nu;
  m.rho = model->ghrl_rho;
  m.sigma = model->ghrl_sigma;
  m.ghrl_c0 = fmaf(-0.5f, m.nu, -m.mu / 9.f);  // IEEE division and fused multiply-add: the device's own value
  for (int k = 0; k < 3; k++) m.fdir[k] = model->field_dir[k];
  m.elecA = model->elecA;
  m.elecP = model->elecP;
  m.flip = model->flip_move != 0;
  m.field_on = (model->elecA != 0 || model->elecP != 0);
  m.n_surf = model->n_surfaces;
  for (int s = 0; s < model->n_surfaces; s++) {
    m.anch_type[s] = model->anch_type[s];
    m.anch_W[s] = model->anch_W[s];
    easy_axis(model->anch_theta[s], model->anch_phi[s], m.anch_lab[s]);
  }
  PlainLattice L;
  L.nx = R.nx;
  L.ny = R.ny;
  L.nz = R.nz;
  L.periodic[0] = R.periodic[0] != 0;
  L.periodic[1] = R.periodic[1] != 0;
  L.periodic[2] = R.geometry == MCL_GEOM_SLAB ? 0 : R.periodic[2] != 0;
  L.n_sites = n_sites;
  const int geo = R.geometry == MCL_GEOM_SLAB ? GEO_SLAB : GEO_BULK;
  const int n_slots = (int)((n_sites + kSitesPerSlot - 1) / kSitesPerSlot);
  cudaStream_t st = (cudaStream_t)stream;

  if (m.potential == POT_GHRL)
    launch_observe_static<POT_GHRL>(geo, n_slots, m, L, R.elecE, d_ni, scratch, st);
  else if (m.potential == POT_PEAR)
    launch_observe_static<POT_PEAR>(geo, n_slots, m, L, R.elecE, d_ni, scratch, st);
  else
    launch_observe_static<POT_LL>(geo, n_slots, m, L, R.elecE, d_ni, scratch, st);
  CK_STATIC(cudaGetLastError());
  ObsRecord *rec = (ObsRecord *)(scratch + kRecordOffset);
  k_observe_static_finalize<<<1, kThreads, 0, st>>>(n_slots, (double)n_sites, (double)R.ang_var, scratch, rec);
  CK_STATIC(cudaGetLastError());
  ObsRecord o;
  CK_STATIC(cudaMemcpyAsync(&o, rec, sizeof o, cudaMemcpyDeviceToHost, st));
  CK_STATIC(cudaStreamSynchronize(st));
  memcpy(out, &o, sizeof o);
  return MCL_OK;
}
