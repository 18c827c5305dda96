// C-ABI implementation: engine lifetime, device buffers, uploads/downloads and the sweep loop.
//
// Replaces the device-side half of EvolveNGPU (src/evolve.cu): the per-run allocations of
// src/evolve_thermal.cu:50-66, the first-call set-up of Monte_Carlo_Step_GPU (src/evolve.cu:319-404, device
// function pointers chosen by name -> template dispatch here), the 8 launches + reduction + host read-back per
// sweep (src/evolve.cu:406-440 -> launches only, ang_var adapted on the device), and energy_calculator_GPU
// (src/evolve.cu:442-478 -> FP64 reductions on the device, fused with the Q tensor).
#include "engine.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "fused.h"

namespace mcl {

static thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t err, const char *what) {
  return fail(err == cudaErrorMemoryAllocation ? MCL_ERR_NOMEM : MCL_ERR_CUDA, "%s: %s (%s)", what,
              cudaGetErrorString(err), cudaGetErrorName(err));
}

#define CK(call)                                         \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Lab easy axis of an anchoring, anchoring.cpp:19-24 (float, host libm, as in the reference).
static void lab_axis(float theta_deg, float phi_deg, float out[3]) {
  const float toRad = (float)(M_PI / 180);
  out[0] = sinf(toRad * theta_deg) * cosf(toRad * phi_deg);
  out[1] = sinf(toRad * theta_deg) * sinf(toRad * phi_deg);
  out[2] = cosf(toRad * theta_deg);
}

// Sphere geometry, src/geometry_sphere.cpp:32-58: centre (nx/2, ny/2, nz/2) by integer division, bulk for
// r < nz/2 - 1, one surface layer (radial normal) for r < nz/2 + 1, empty outside.
static void sphere_geometry(int nx, int ny, int nz, int *pt, float *ns) {
  const float Hx = nx / 2, Hy = ny / 2, Hz = nz / 2;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const long long idx = i + (long long)nx * (j + (long long)ny * k);
        float Rx = i - Hx, Ry = j - Hy, Rz = k - Hz;
        float radius = sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
        ns[3 * idx] = ns[3 * idx + 1] = ns[3 * idx + 2] = 0.f;
        if (radius < Hz - 1) {
          pt[idx] = 1;
        } else if (radius < Hz + 1) {
          pt[idx] = 2;
          ns[3 * idx + 0] = Rx / radius;
          ns[3 * idx + 1] = Ry / radius;
          ns[3 * idx + 2] = Rz / radius;
        } else {
          pt[idx] = 0;
        }
      }
}

static int build_table(BlockTable &t, const std::vector<long long> &items, int threads) {
  std::vector<int> rep, first;
  std::vector<long long> base;
  for (size_t r = 0; r < items.size(); r++) {
    first.push_back((int)rep.size());
    for (long long b = 0; b < items[r]; b += threads) {
      rep.push_back((int)r);
      base.push_back(b);
    }
  }
  first.push_back((int)rep.size());
  t.n_blocks = (int)rep.size();
  CK(cudaMalloc(&t.first, first.size() * sizeof(int)));
  CK(cudaMemcpy(t.first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (t.n_blocks) {
    CK(cudaMalloc(&t.rep, rep.size() * sizeof(int)));
    CK(cudaMalloc(&t.base, base.size() * sizeof(long long)));
    CK(cudaMemcpy(t.rep, rep.data(), rep.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.base, base.data(), base.size() * sizeof(long long), cudaMemcpyHostToDevice));
  }
  return MCL_OK;
}

static void free_table(BlockTable &t) {
  cudaFree(t.rep);
  cudaFree(t.base);
  cudaFree(t.first);
  t = BlockTable();
}

static int ensure_series(mcl_engine *e, int rows) {
  if (rows <= e->series_cap) return MCL_OK;
  int cap = std::max(rows, std::max(64, 2 * e->series_cap));
  ObsRecord *p = nullptr;
  CK(cudaMalloc(&p, (size_t)cap * e->n_rep * sizeof(ObsRecord)));
  if (e->d_series) {
    CK(cudaMemcpyAsync(p, e->d_series, (size_t)e->series_cap * e->n_rep * sizeof(ObsRecord), cudaMemcpyDeviceToDevice,
                       e->stream));
    CK(cudaStreamSynchronize(e->stream));
    cudaFree(e->d_series);
  }
  e->d_series = p;
  e->series_cap = cap;
  return MCL_OK;
}

// Error words of the fused sweep (TMA waits) and the learned sweep (tensor-core waits); synchronises.
static int kernel_errors(mcl_engine *e) {
  const int rc = fused_check_error(e);
  return rc ? rc : learned_check_error(e);
}

// Captured sweep graphs hold kernel arguments (work items, buffers, series, test hooks): drop them whenever one of
// those changes.
static void drop_graphs(mcl_engine *e) {
  for (int m = 0; m < 2; m++) {
    if (e->graph[m]) cudaGraphExecDestroy(e->graph[m]);
    e->graph[m] = nullptr;
  }
  e->graph_series = nullptr;
  if (e->graph_io) cudaGraphExecDestroy(e->graph_io);
  e->graph_io = nullptr;
  e->graph_io_series = e->graph_io_stage = nullptr;
}

// Sweeps per captured graph: one for the in-place colour passes, two for the ping-pong fused kernel (one per
// buffer parity, so that a replay leaves the buffers where it found them).
static int graph_sweeps(const mcl_engine *e) { return fused_is_pass_plan(e) ? 1 : 2; }

// Captures graph_sweeps(e) sweeps starting from buffer e->cur as a graph. Every per-sweep quantity the kernels use
// (sweep counter, temperatures, ang_var, series length) lives in device memory, so a replay does exactly what the
// same direct calls would.
static int capture_graph(mcl_engine *e, int m) {
  if (e->graph[m]) cudaGraphExecDestroy(e->graph[m]);
  e->graph[m] = nullptr;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const int cur0 = e->cur;
  const long long l0 = e->launches;
  int rc = MCL_OK;
  for (int s = 0; s < graph_sweeps(e) && !rc; s++) rc = fused_sweep(e, m != 0, nullptr, nullptr);
  const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
  e->cur = cur0;
  e->launches = l0;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
  const cudaError_t ie = cudaGraphInstantiate(&e->graph[m], g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    e->graph[m] = nullptr;
    return cuda_fail(ie, "cudaGraphInstantiate");
  }
  e->graph_cur[m] = cur0;
  if (m) e->graph_series = e->d_series;
  return MCL_OK;
}

static int refresh_ghosts(mcl_engine *e) {
  if (!e->ghosts_dirty) return MCL_OK;
  CK(launch_refresh_ghosts(e->ctx(), 0, 0));
  e->ghosts_dirty = false;
  return MCL_OK;
}

}  // namespace mcl

using namespace mcl;

extern "C" {

const char *mcl_last_error(void) { return g_err.c_str(); }
const char *mcl_version(void) { return "mclics_b200 0.1 (sm_100a)"; }

int mcl_create(const mcl_model *model, const mcl_replica *replicas, int n_replicas, int schedule, mcl_engine **out) {
  if (!model || !replicas || !out || n_replicas < 1) return fail(MCL_ERR_ARG, "mcl_create: null argument or no replicas");
  *out = nullptr;
  if (schedule < MCL_SCHED_REF8 || schedule > MCL_SCHED_CHECKER2_SIMPLE)
    return fail(MCL_ERR_ARG, "mcl_create: unknown schedule %d", schedule);
  if (model->potential < MCL_POT_LL || model->potential > MCL_POT_PEAR)
    return fail(MCL_ERR_ARG, "mcl_create: unknown potential %d", model->potential);
  if (model->n_surfaces < 0 || model->n_surfaces > MCL_MAX_SURFACES)
    return fail(MCL_ERR_ARG, "mcl_create: n_surfaces %d outside 0..%d", model->n_surfaces, MCL_MAX_SURFACES);
  for (int s = 0; s < model->n_surfaces; s++)
    if (model->anch_type[s] < MCL_ANCH_HOMEOTROPIC || model->anch_type[s] > MCL_ANCH_FG_GHRL)
      return fail(MCL_ERR_ARG, "mcl_create: unknown anchoring type %d of surface %d", model->anch_type[s], s);
  int geo_class = -1;
  for (int r = 0; r < n_replicas; r++) {
    const mcl_replica &R = replicas[r];
    if (R.nx < 1 || R.ny < 1 || R.nz < 1) return fail(MCL_ERR_ARG, "replica %d: grid sizes must be >= 1", r);
    if ((long long)R.nx * R.ny * R.nz >= (1ll << 32)) return fail(MCL_ERR_ARG, "replica %d: more than 2^32 sites", r);
    int g;
    switch (R.geometry) {
      case MCL_GEOM_BULK: g = GEO_BULK; break;
      case MCL_GEOM_SLAB: g = GEO_SLAB; break;
      case MCL_GEOM_SPHERE:
      case MCL_GEOM_CUSTOM: g = GEO_PT; break;
      default: return fail(MCL_ERR_ARG, "replica %d: unknown geometry %d", r, R.geometry);
    }
    if (geo_class >= 0 && g != geo_class)
      return fail(MCL_ERR_ARG, "replicas of one engine must share the geometry kind (bulk / slab / sphere+custom)");
    geo_class = g;
    int per[3] = {R.periodic[0] != 0, R.periodic[1] != 0, R.periodic[2] != 0};
    if (R.geometry == MCL_GEOM_SLAB) per[2] = 0;
    if (R.geometry == MCL_GEOM_SPHERE) per[0] = per[1] = per[2] = 0;
    const int n[3] = {R.nx, R.ny, R.nz};
    for (int a = 0; a < 3; a++)
      if (per[a] && n[a] % 2)
        return fail(MCL_ERR_ARG,
                    "replica %d: periodic boundary along %c requires an even number of sites (N%c = %d); the "
                    "checkerboard update needs it",
                    r, "xyz"[a], "xyz"[a], n[a]);
    if (R.geometry == MCL_GEOM_SLAB && model->n_surfaces < 2)
      return fail(MCL_ERR_ARG, "slab geometry needs anchoring for surfaces 0 and 1");
    if (R.geometry == MCL_GEOM_SPHERE && model->n_surfaces < 1)
      return fail(MCL_ERR_ARG, "sphere geometry needs anchoring for surface 0");
    if (!(R.T >= 0.f)) return fail(MCL_ERR_ARG, "replica %d: temperature must be >= 0", r);
  }
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return fail(MCL_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(ce));
  cudaDeviceProp prop;
  ce = cudaGetDeviceProperties(&prop, dev);
  if (ce != cudaSuccess) return fail(MCL_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(ce));
  if (prop.major != 10) return fail(MCL_ERR_NO_DEVICE, "this library is built for sm_100 (B200); device is sm_%d%d", prop.major, prop.minor);

  mcl_engine *e = new mcl_engine();
  e->device = dev;
  e->model_in = *model;
  e->schedule = schedule;
  e->geo = geo_class;
  e->n_rep = n_replicas;
  e->rep_in.assign(replicas, replicas + n_replicas);
  ModelDev &m = e->model;
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
    lab_axis(model->anch_theta[s], model->anch_phi[s], m.anch_lab[s]);
  }

  // layouts
  long long off = 0, soff = 0;
  e->desc.resize(n_replicas);
  std::vector<RepState> st(n_replicas);
  e->host_pt.clear();
  bool need_pt = geo_class == GEO_PT;
  for (int r = 0; r < n_replicas; r++) {
    const mcl_replica &R = replicas[r];
    RepDesc &D = e->desc[r];
    memset(&D, 0, sizeof D);
    D.nx = R.nx;
    D.ny = R.ny;
    D.nz = R.nz;
    D.hp = (((R.nx + 1) / 2 + 3) / 4) * 4 + 2 * GH;
    D.px = 2 * D.hp;
    D.py = R.ny + 2 * GY;
    D.geo = geo_class;
    D.periodic[0] = R.periodic[0] != 0;
    D.periodic[1] = R.periodic[1] != 0;
    D.periodic[2] = R.periodic[2] != 0;
    if (R.geometry == MCL_GEOM_SLAB) D.periodic[2] = 0;
    if (R.geometry == MCL_GEOM_SPHERE) D.periodic[0] = D.periodic[1] = D.periodic[2] = 0;
    D.comp = (long long)R.nz * D.py * D.px;
    D.off = off;
    off += 3 * D.comp;
    off = (off + 31) / 32 * 32;  // 128-byte alignment of every replica
    D.site_off = soff;
    const long long N = (long long)R.nx * R.ny * R.nz;
    soff += N;
    D.seed = R.seed;
    D.n_valid = (double)N;
    D.zslab = 0;
    D.zoff = 0;
    D.nzg = R.nz;
    st[r].T = R.T;
    st[r].elecE = R.elecE;
    st[r].ang_var = R.ang_var;
    st[r].pad = 0.f;
    st[r].acc = 0;
    e->max_sites = std::max(e->max_sites, N);
  }
  e->dir_floats = off;
  e->n_sites = soff;

  auto cleanup_fail = [&](int code) {
    mcl_destroy(e);
    return code;
  };
#define CKC(call)                                                  \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return cleanup_fail(cuda_fail(e_, #call)); \
  } while (0)

  CKC(cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking));
  e->stream = e->own_stream;
  CKC(cudaMalloc(&e->d_dir[0], (size_t)e->dir_floats * sizeof(float)));
  CKC(cudaMemsetAsync(e->d_dir[0], 0, (size_t)e->dir_floats * sizeof(float), e->stream));
  CKC(cudaMalloc(&e->d_stage, (size_t)e->max_sites * 3 * sizeof(float)));
  CKC(cudaMalloc(&e->d_desc, n_replicas * sizeof(RepDesc)));
  CKC(cudaMalloc(&e->d_state, n_replicas * sizeof(RepState)));
  CKC(cudaMalloc(&e->d_sweep, sizeof(unsigned long long)));
  CKC(cudaMalloc(&e->d_done, sizeof(unsigned int)));
  CKC(cudaMalloc(&e->d_series_len, sizeof(int)));
  CKC(cudaMalloc(&e->d_probe_len, sizeof(int)));
  CKC(cudaMalloc(&e->d_probe, n_replicas * sizeof(ObsRecord)));
  CKC(cudaMemsetAsync(e->d_sweep, 0, sizeof(unsigned long long), e->stream));
  CKC(cudaMemsetAsync(e->d_done, 0, sizeof(unsigned int), e->stream));
  CKC(cudaMemsetAsync(e->d_series_len, 0, sizeof(int), e->stream));
  CKC(cudaMemsetAsync(e->d_probe_len, 0, sizeof(int), e->stream));
  if (need_pt) {
    CKC(cudaMalloc(&e->d_pt, (size_t)e->n_sites));
    CKC(cudaMalloc(&e->d_nrm, (size_t)e->n_sites * 3 * sizeof(float)));
    e->host_pt.assign((size_t)e->n_sites, 1);
    std::vector<float> ns((size_t)e->n_sites * 3, 0.f);
    e->geometry_set = true;
    for (int r = 0; r < n_replicas; r++) {
      const RepDesc &D = e->desc[r];
      if (replicas[r].geometry == MCL_GEOM_SPHERE)
        sphere_geometry(D.nx, D.ny, D.nz, &e->host_pt[D.site_off], &ns[3 * D.site_off]);
      else
        e->geometry_set = false;  // custom: mcl_set_geometry required before sweeping
    }
    std::vector<uint8_t> p8(e->host_pt.begin(), e->host_pt.end());
    CKC(cudaMemcpy(e->d_pt, p8.data(), p8.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(e->d_nrm, ns.data(), ns.size() * sizeof(float), cudaMemcpyHostToDevice));
    for (int r = 0; r < n_replicas; r++) {
      const RepDesc &D = e->desc[r];
      long long nv = 0;
      for (long long q = 0; q < (long long)D.nx * D.ny * D.nz; q++) nv += e->host_pt[D.site_off + q] != 0;
      e->desc[r].n_valid = (double)nv;
    }
  }
  CKC(cudaMemcpy(e->d_desc, e->desc.data(), n_replicas * sizeof(RepDesc), cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(e->d_state, st.data(), n_replicas * sizeof(RepState), cudaMemcpyHostToDevice));

  std::vector<long long> half, boxes, sites;
  for (auto &D : e->desc) {
    half.push_back((long long)((D.nx + 1) / 2) * D.ny * D.nz);
    boxes.push_back((long long)((D.nx + 1) / 2) * ((D.ny + 1) / 2) * ((D.nz + 1) / 2));
    sites.push_back((long long)D.nx * D.ny * D.nz);
  }
  int rc;
  if ((rc = build_table(e->half, half, kThreads)) != MCL_OK) return cleanup_fail(rc);
  if ((rc = build_table(e->boxes, boxes, kThreads)) != MCL_OK) return cleanup_fail(rc);
  if ((rc = build_table(e->sites, sites, kThreads)) != MCL_OK) return cleanup_fail(rc);
  CKC(cudaMalloc(&e->d_partials, (size_t)std::max(1, e->sites.n_blocks) * kPartials * sizeof(double)));

  // directors start at (0, 0, 1) (the reference's value for unset sites)
  {
    std::vector<float> aos((size_t)e->max_sites * 3);
    for (long long q = 0; q < e->max_sites; q++) {
      aos[3 * q] = 0.f;
      aos[3 * q + 1] = 0.f;
      aos[3 * q + 2] = 1.f;
    }
    CKC(cudaMemcpy(e->d_stage, aos.data(), aos.size() * sizeof(float), cudaMemcpyHostToDevice));
    for (int r = 0; r < n_replicas; r++) CKC(launch_unpack(e->ctx(), r, e->desc[r], e->d_stage));
  }
  if (schedule == MCL_SCHED_CHECKER2 && fused_supported(e)) {
    if ((rc = fused_create(e)) != MCL_OK) return cleanup_fail(rc);
  }
  e->ghosts_dirty = true;
  if ((rc = refresh_ghosts(e)) != MCL_OK) return cleanup_fail(rc);
  CKC(cudaStreamSynchronize(e->stream));
#undef CKC
  *out = e;
  return MCL_OK;
}

int mcl_destroy(mcl_engine *e) {
  if (!e) return MCL_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graphs(e);
  if (e->fused) fused_destroy(e);
  free_table(e->half);
  free_table(e->boxes);
  free_table(e->sites);
  cudaFree(e->d_dir[0]);
  cudaFree(e->d_dir[1]);
  cudaFree(e->d_mlp);
  cudaFree(e->d_mlp_tc);
  cudaFree(e->d_lerr);
  cudaFree(e->d_xpart);
  cudaFree(e->d_pt);
  cudaFree(e->d_nrm);
  cudaFree(e->d_stage);
  cudaFree(e->d_desc);
  cudaFree(e->d_state);
  cudaFree(e->d_sweep);
  cudaFree(e->d_done);
  cudaFree(e->d_series_len);
  cudaFree(e->d_series);
  cudaFree(e->d_probe);
  cudaFree(e->d_probe_len);
  cudaFree(e->d_partials);
  cudaFree(e->d_dec);
  cudaFreeHost(e->h_io);
  for (cudaEvent_t ev : e->ev_pool) cudaEventDestroy(ev);
  if (e->own_stream) cudaStreamDestroy(e->own_stream);
  delete e;
  return MCL_OK;
}

static int check_rep(mcl_engine *e, int r, bool allow_all) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (allow_all && r == -1) return MCL_OK;
  if (r < 0 || r >= e->n_rep) return fail(MCL_ERR_ARG, "replica %d outside 0..%d", r, e->n_rep - 1);
  return MCL_OK;
}

int mcl_set_geometry(mcl_engine *e, int replica, const int *pt, const float *normals) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (e->geo != GEO_PT) return fail(MCL_ERR_STATE, "mcl_set_geometry: only sphere and custom replicas take point types");
  if (!pt || !normals) return fail(MCL_ERR_ARG, "mcl_set_geometry: null array");
  const RepDesc &D = e->desc[replica];
  const long long N = (long long)D.nx * D.ny * D.nz;
  std::vector<uint8_t> p8(N);
  long long nv = 0;
  for (long long q = 0; q < N; q++) {
    if (pt[q] < 0 || pt[q] > 1 + e->model.n_surf)
      return fail(MCL_ERR_ARG, "point type %d at site %lld: valid are 0, 1 and 2..%d", pt[q], q, 1 + e->model.n_surf);
    p8[q] = (uint8_t)pt[q];
    e->host_pt[D.site_off + q] = pt[q];
    nv += pt[q] != 0;
  }
  if (nv == 0) return fail(MCL_ERR_ARG, "mcl_set_geometry: no non-empty site");
  CK(cudaMemcpyAsync(e->d_pt + D.site_off, p8.data(), N, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(e->d_nrm + 3 * D.site_off, normals, N * 3 * sizeof(float), cudaMemcpyHostToDevice, e->stream));
  e->desc[replica].n_valid = (double)nv;
  CK(cudaMemcpyAsync(e->d_desc + replica, &e->desc[replica], sizeof(RepDesc), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->geometry_set = true;
  return MCL_OK;
}

int mcl_upload_directors(mcl_engine *e, int replica, const float *ni) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (!ni) return fail(MCL_ERR_ARG, "mcl_upload_directors: null array");
  const RepDesc &D = e->desc[replica];
  const long long N = (long long)D.nx * D.ny * D.nz;
  for (long long q = 0; q < N; q++) {
    if (e->geo == GEO_PT && e->host_pt[D.site_off + q] == 0) continue;
    const float x = ni[3 * q], y = ni[3 * q + 1], z = ni[3 * q + 2];
    const float n2 = x * x + y * y + z * z;
    if (!isfinite(x) || !isfinite(y) || !isfinite(z) || !(n2 > 1e-12f))
      return fail(MCL_ERR_NONFINITE, "director of site %lld is not finite or has zero length (%g, %g, %g)", q, x, y, z);
  }
  CK(cudaMemcpyAsync(e->d_stage, ni, N * 3 * sizeof(float), cudaMemcpyHostToDevice, e->stream));
  CK(launch_unpack(e->ctx(), replica, D, e->d_stage));
  e->ghosts_dirty = true;
  if ((rc = refresh_ghosts(e))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return MCL_OK;
}

int mcl_random_directors(mcl_engine *e, int replica, unsigned long long seed) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  CK(launch_random_ic(e->ctx(), e->desc[replica], seed));
  e->ghosts_dirty = true;
  if ((rc = refresh_ghosts(e))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return kernel_errors(e);
}

int mcl_download_directors(mcl_engine *e, int replica, float *ni) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (!ni) return fail(MCL_ERR_ARG, "mcl_download_directors: null array");
  const RepDesc &D = e->desc[replica];
  const long long N = (long long)D.nx * D.ny * D.nz;
  CK(launch_pack(e->ctx(), replica, D, e->d_stage));
  CK(cudaMemcpyAsync(ni, e->d_stage, N * 3 * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return kernel_errors(e);
}

static int set_state_field(mcl_engine *e, int replica, size_t offset, float v) {
  int rc = check_rep(e, replica, true);
  if (rc) return rc;
  for (int r = 0; r < e->n_rep; r++) {
    if (replica != -1 && r != replica) continue;
    CK(cudaMemcpyAsync((char *)(e->d_state + r) + offset, &v, sizeof(float), cudaMemcpyHostToDevice, e->stream));
  }
  CK(cudaStreamSynchronize(e->stream));
  return MCL_OK;
}

int mcl_set_temperature(mcl_engine *e, int replica, float T) {
  if (!(T >= 0.f)) return fail(MCL_ERR_ARG, "temperature must be >= 0 (got %g)", T);
  return set_state_field(e, replica, offsetof(RepState, T), T);
}
int mcl_set_field(mcl_engine *e, int replica, float elecE) {
  if (!isfinite(elecE)) return fail(MCL_ERR_ARG, "field magnitude must be finite");
  return set_state_field(e, replica, offsetof(RepState, elecE), elecE);
}
int mcl_set_ang_var(mcl_engine *e, int replica, float v) {
  if (!(v > 0.f) || !isfinite(v)) return fail(MCL_ERR_ARG, "ang_var must be > 0 (got %g)", v);
  return set_state_field(e, replica, offsetof(RepState, ang_var), v);
}

int mcl_get_ang_var(mcl_engine *e, int replica, float *v) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (!v) return fail(MCL_ERR_ARG, "null output");
  CK(cudaMemcpyAsync(v, (char *)(e->d_state + replica) + offsetof(RepState, ang_var), sizeof(float),
                     cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return MCL_OK;
}

int mcl_set_sweep_counter(mcl_engine *e, unsigned long long sweep) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaMemcpyAsync(e->d_sweep, &sweep, sizeof sweep, cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return MCL_OK;
}

int mcl_get_sweep_counter(mcl_engine *e, unsigned long long *sweep) {
  if (!e || !sweep) return fail(MCL_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(sweep, e->d_sweep, sizeof *sweep, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return MCL_OK;
}

static int sweeps_run(mcl_engine *e, int n, int measure);

int mcl_sweeps(mcl_engine *e, int n, int measure) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (n < 0) return fail(MCL_ERR_ARG, "negative sweep count");
  if (e->zslab) return fail(MCL_ERR_STATE, "mcl_sweeps: a z-slab engine sweeps through the mcl_zslab_* calls");
  if (!e->geometry_set) return fail(MCL_ERR_STATE, "custom geometry: call mcl_set_geometry before sweeping");
  if (n == 0) return MCL_OK;
  if (!e->d_mlp || e->mix_period <= 1) return sweeps_run(e, n, measure);
  // Mixture of the learned and the plain sweep: one learned sweep after every mix_period - 1 plain ones, counted
  // across calls. Both sweeps are exact Metropolis(-Hastings) kernels of the same distribution, so a fixed cycle
  // of them is one too. The plain sweeps run with the learned weights set aside.
  while (n > 0) {
    const int until_learned = e->mix_period - 1 - e->mix_phase;
    const bool learned = until_learned == 0;
    const int run = learned ? 1 : std::min(n, until_learned);
    MlpDev *weights = e->d_mlp;
    if (!learned) e->d_mlp = nullptr;
    const int rc = sweeps_run(e, run, measure);
    e->d_mlp = weights;
    if (rc) return rc;
    e->mix_phase = (e->mix_phase + run) % e->mix_period;
    n -= run;
  }
  return MCL_OK;
}

int mcl_set_proposal_mix(mcl_engine *e, int period) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (period < 1) return fail(MCL_ERR_ARG, "mcl_set_proposal_mix: the period must be >= 1 (got %d)", period);
  e->mix_period = period;
  e->mix_phase = 0;
  return MCL_OK;
}

static int sweeps_run(mcl_engine *e, int n, int measure) {
  int rc;
  if (measure && (rc = ensure_series(e, e->series_len + n))) return rc;
  const bool use_fused = e->fused && !e->record_dec && !e->d_mlp;
  if (use_fused && (rc = refresh_ghosts(e))) return rc;
  const int per_graph = use_fused ? graph_sweeps(e) : 2;
  if (use_fused && e->use_graphs && !e->profile && n >= per_graph) {
    const int m = measure ? 1 : 0;
    if (!e->graph[m] || (m && e->graph_series != (const void *)e->d_series)) {
      if ((rc = capture_graph(e, m))) return rc;
    }
    if (e->cur != e->graph_cur[m]) {  // one direct sweep brings the buffers to the graph's parity
      if ((rc = fused_sweep(e, measure != 0, nullptr, nullptr))) return rc;
      if (measure) e->series_len++;
      n--;
    }
    for (; n >= per_graph; n -= per_graph) {
      CK(cudaGraphLaunch(e->graph[m], e->stream));
      e->launches += per_graph * fused_launches_per_sweep(e);
      if (measure) e->series_len += per_graph;
    }
  }
  for (int s = 0; s < n; s++) {
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (e->profile) {
      while (e->ev_pool.size() < e->ev_used + 2) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev));
        e->ev_pool.push_back(ev);
      }
      ev0 = e->ev_pool[e->ev_used];
      ev1 = e->ev_pool[e->ev_used + 1];
      e->ev_used += 2;
    }
    if (use_fused) {
      if ((rc = fused_sweep(e, measure != 0, ev0, ev1))) return rc;
    } else {
      LaunchCtx c = e->ctx();
      if (ev0) CK(cudaEventRecord(ev0, e->stream));
      if (e->d_mlp && e->mlp_tc && e->learned_pass && e->fused) {  // colour passes on streamed planes
        const LearnedMlp lm{e->d_mlp, e->d_mlp_tc, e->d_lerr, e->mlp_tc};
        LearnedPassView v;
        if ((rc = refresh_ghosts(e))) return rc;  // the passes read ghost cells and keep them current
        if ((rc = fused_learned_view(e, &v))) return rc;
        CK(launch_learned_pass(c, e->geo, v, lm, e->kappa_max, measure ? 1 : 0, e->d_dir[e->cur], e->cur));
        e->launches += 2;
        if (ev1) CK(cudaEventRecord(ev1, e->stream));
        BlockTable t;
        t.first = v.first;
        CK(launch_finalize(c, t, v.partials, measure ? 1 : 0, e->d_series, e->d_series_len, e->d_done));
        e->launches++;
        if (measure) e->series_len++;
        continue;
      }
      if (e->d_mlp) {  // observables fused into the two colour kernels, finalised over the same block table
        const LearnedMlp lm{e->d_mlp, e->d_mlp_tc, e->d_lerr, e->mlp_tc};
        CK(launch_sweep_learned(c, e->geo, e->half, lm, e->kappa_max, measure ? 1 : 0, e->d_partials));
        e->launches += 2;
        if (ev1) CK(cudaEventRecord(ev1, e->stream));
        CK(launch_finalize(c, e->half, e->d_partials, measure ? 1 : 0, e->d_series, e->d_series_len, e->d_done));
        e->launches++;
        e->ghosts_dirty = true;
        if (measure) e->series_len++;
        continue;
      } else if (e->schedule == MCL_SCHED_REF8) {
        CK(launch_sweep_ref8(c, e->geo, e->boxes));
        e->launches += 8;
      } else {
        CK(launch_sweep_checker2_simple(c, e->geo, e->half));
        e->launches += 2;
      }
      if (ev1) CK(cudaEventRecord(ev1, e->stream));
      if (measure) {
        CK(launch_observe(c, e->geo, e->sites, e->d_partials));
        e->launches++;
      }
      CK(launch_finalize(c, e->sites, e->d_partials, measure ? 1 : 0, e->d_series, e->d_series_len, e->d_done));
      e->launches++;
      e->ghosts_dirty = true;
    }
    if (measure) e->series_len++;
  }
  return MCL_OK;
}

static void to_public(const ObsRecord &o, mcl_observables *p);

int mcl_sweeps_io(mcl_engine *e, int n, const float *T, mcl_observables *out) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (n < 1) return fail(MCL_ERR_ARG, "mcl_sweeps_io: n must be >= 1 (got %d)", n);
  if (!out) return fail(MCL_ERR_ARG, "null output");
  if (e->zslab) return fail(MCL_ERR_STATE, "mcl_sweeps_io: a z-slab engine sweeps through the mcl_zslab_* calls");
  if (T)
    for (int r = 0; r < e->n_rep; r++)
      if (!(T[r] >= 0.f) || !isfinite(T[r]))
        return fail(MCL_ERR_ARG, "temperature of replica %d must be finite and >= 0 (got %g)", r, T[r]);
  // mapped pinned staging: two error words, the temperatures, the records (64-byte aligned parts)
  const size_t t_off = 64, rec_off = t_off + ((size_t)e->n_rep * sizeof(float) + 63) / 64 * 64;
  const size_t rec_bytes = (size_t)n * e->n_rep * sizeof(ObsRecord), need = rec_off + rec_bytes;
  if (e->io_inflight || need > e->h_io_bytes) CK(cudaStreamSynchronize(e->stream));
  e->io_inflight = false;
  if (need > e->h_io_bytes) {
    cudaFreeHost(e->h_io);
    e->h_io = nullptr;
    e->d_io = nullptr;
    e->h_io_bytes = 0;
    CK(cudaHostAlloc(&e->h_io, need, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(&e->d_io, e->h_io, 0));
    e->h_io_bytes = need;
  }
  unsigned *words = (unsigned *)e->h_io;
  float *hT = (float *)((char *)e->h_io + t_off);
  ObsRecord *rec = (ObsRecord *)((char *)e->h_io + rec_off);
  char *dio = (char *)e->d_io;
  words[0] = words[1] = 0;
  int rc;
  // One measured sweep of a colour-pass plan with graphs on: the whole step is one captured graph (input kernel,
  // the sweep's kernels, output kernel reading the newest record), captured again when a buffer it uses moves.
  const bool use_fused = e->fused && !e->record_dec && !e->d_mlp;
  if (T && n == 1 && use_fused && e->use_graphs && !e->profile && fused_is_pass_plan(e)) {
    if ((rc = ensure_series(e, e->series_len + 1))) return rc;
    if ((rc = refresh_ghosts(e))) return rc;
    if (!e->graph_io || e->graph_io_series != (const void *)e->d_series || e->graph_io_stage != e->d_io) {
      if (e->graph_io) cudaGraphExecDestroy(e->graph_io);
      e->graph_io = nullptr;
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
      const long long l0 = e->launches;
      cudaError_t ce = launch_io_in(e->stream, e->d_state, (const float *)(dio + t_off), e->n_rep);
      rc = ce == cudaSuccess ? fused_sweep(e, true, nullptr, nullptr) : MCL_OK;
      if (ce == cudaSuccess && !rc)
        ce = launch_io_out(e->stream, e->d_series, 0, e->d_series_len, 1, e->n_rep, (ObsRecord *)(dio + rec_off),
                           fused_error_word(e), e->d_lerr, (unsigned *)dio);
      const cudaError_t ee = cudaStreamEndCapture(e->stream, &g);
      e->launches = l0;
      if (rc || ce != cudaSuccess || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (rc) return rc;
        return cuda_fail(ce != cudaSuccess ? ce : ee, "mcl_sweeps_io: graph capture");
      }
      const cudaError_t ie = cudaGraphInstantiate(&e->graph_io, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        e->graph_io = nullptr;
        return cuda_fail(ie, "cudaGraphInstantiate");
      }
      e->graph_io_series = e->d_series;
      e->graph_io_stage = e->d_io;
    }
    memcpy(hT, T, (size_t)e->n_rep * sizeof(float));
    e->io_inflight = true;
    CK(cudaGraphLaunch(e->graph_io, e->stream));
    e->launches += 2 + fused_launches_per_sweep(e);
    e->series_len++;
  } else {
    if (T) {
      memcpy(hT, T, (size_t)e->n_rep * sizeof(float));
      e->io_inflight = true;
      CK(launch_io_in(e->stream, e->d_state, (const float *)(dio + t_off), e->n_rep));
      e->launches++;
    }
    const int first = e->series_len;
    if ((rc = mcl_sweeps(e, n, 1))) return rc;
    e->io_inflight = true;
    CK(launch_io_out(e->stream, e->d_series, first, nullptr, n, e->n_rep, (ObsRecord *)(dio + rec_off),
                     fused_error_word(e), e->d_lerr, (unsigned *)dio));
    e->launches++;
  }
  CK(cudaStreamSynchronize(e->stream));
  e->io_inflight = false;
  if ((rc = fused_report_error(e, words[0]))) return rc;
  if ((rc = learned_report_error(e, words[1]))) return rc;
  for (size_t i = 0; i < (size_t)n * e->n_rep; i++) to_public(rec[i], out + i);
  return MCL_OK;
}

int mcl_set_stream(mcl_engine *e, void *stream) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaStreamSynchronize(e->stream));
  e->stream = stream ? (cudaStream_t)stream : e->own_stream;
  return MCL_OK;
}

int mcl_profile(mcl_engine *e, int enable) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  e->profile = enable != 0;
  return MCL_OK;
}

int mcl_profile_read(mcl_engine *e, double *ms, long long *sweeps, long long *launches) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaStreamSynchronize(e->stream));
  for (size_t k = 0; k + 1 < e->ev_used; k += 2) {
    float t = 0;
    CK(cudaEventElapsedTime(&t, e->ev_pool[k], e->ev_pool[k + 1]));
    e->prof_ms += t;
    e->prof_sweeps++;
  }
  e->ev_used = 0;
  if (ms) *ms = e->prof_ms;
  if (sweeps) *sweeps = e->prof_sweeps;
  if (launches) *launches = e->launches;
  return MCL_OK;
}

int mcl_series_length(mcl_engine *e, int *n) {
  if (!e || !n) return fail(MCL_ERR_ARG, "null argument");
  *n = e->series_len;
  return MCL_OK;
}

static void to_public(const ObsRecord &o, mcl_observables *p) {
  p->energy = o.energy;
  for (int k = 0; k < 6; k++) p->q[k] = o.q[k];
  p->S = o.S;
  for (int k = 0; k < 3; k++) {
    p->director[k] = o.director[k];
    p->nsum[k] = o.nsum[k];
  }
  p->n_valid = o.n_valid;
  p->acceptance = o.acceptance;
  p->ang_var = o.ang_var;
  p->sweep = o.sweep;
}

int mcl_read_series(mcl_engine *e, int replica, int first, int count, mcl_observables *out) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (count < 0 || first < 0 || first + count > e->series_len)
    return fail(MCL_ERR_ARG, "series range [%d, %d) outside the %d records", first, first + count, e->series_len);
  if (count == 0) return MCL_OK;
  if (!out) return fail(MCL_ERR_ARG, "null output");
  std::vector<ObsRecord> rows((size_t)count);
  CK(cudaMemcpy2DAsync(rows.data(), sizeof(ObsRecord), e->d_series + (size_t)first * e->n_rep + replica,
                       (size_t)e->n_rep * sizeof(ObsRecord), sizeof(ObsRecord), count, cudaMemcpyDeviceToHost,
                       e->stream));
  CK(cudaStreamSynchronize(e->stream));
  if ((rc = kernel_errors(e))) return rc;
  for (int i = 0; i < count; i++) to_public(rows[i], out + i);
  return MCL_OK;
}

int mcl_reserve_series(mcl_engine *e, int rows) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (rows < 0) return fail(MCL_ERR_ARG, "mcl_reserve_series: negative row count");
  if (rows <= e->series_cap) return MCL_OK;
  drop_graphs(e);  // captured graphs write the old buffer
  return ensure_series(e, rows);
}

int mcl_clear_series(mcl_engine *e) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaMemsetAsync(e->d_series_len, 0, sizeof(int), e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->series_len = 0;
  return MCL_OK;
}

int mcl_measure(mcl_engine *e, int replica, mcl_observables *out) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (!out) return fail(MCL_ERR_ARG, "null output");
  if (e->zslab) return fail(MCL_ERR_STATE, "mcl_measure: a z-slab engine holds part of a lattice (use mcl_zslab_sums)");
  LaunchCtx c = e->ctx();
  CK(launch_observe(c, e->geo, e->sites, e->d_partials));
  CK(launch_finalize(c, e->sites, e->d_partials, 2, e->d_probe, e->d_probe_len, e->d_done));
  ObsRecord o;
  CK(cudaMemcpyAsync(&o, e->d_probe + replica, sizeof o, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  if ((rc = kernel_errors(e))) return rc;
  to_public(o, out);
  return MCL_OK;
}

int mcl_synchronize(mcl_engine *e) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaStreamSynchronize(e->stream));
  CK(cudaGetLastError());
  return kernel_errors(e);
}

int mcl_debug_wait_limit(mcl_engine *e, long long timeout_ns, int withhold_first_load) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  drop_graphs(e);
  if (!e->fused) return fail(MCL_ERR_STATE, "this engine does not use the fused tiled sweep");
  fused_set_test_hooks(e, timeout_ns, withhold_first_load);
  return MCL_OK;
}

int mcl_set_adaptation(mcl_engine *e, int enable) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaStreamSynchronize(e->stream));
  e->adapt = enable != 0;
  drop_graphs(e);  // captured finalisations hold the flag as an argument
  return MCL_OK;
}

int mcl_set_graphs(mcl_engine *e, int enable) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  CK(cudaStreamSynchronize(e->stream));
  e->use_graphs = enable != 0;
  if (!e->use_graphs) drop_graphs(e);
  return MCL_OK;
}

int mcl_autotune(mcl_engine *e, int trial_sweeps, mcl_tuning *out) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (trial_sweeps < 1 || trial_sweeps > 10000) return fail(MCL_ERR_ARG, "mcl_autotune: trial_sweeps outside 1..10000");
  if (!e->fused || e->record_dec || e->d_mlp || e->zslab)
    return fail(MCL_ERR_STATE, "mcl_autotune: the engine does not run the tiled sweep of whole lattices");
  int rc;
  if ((rc = ensure_series(e, e->series_len + trial_sweeps + 1))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  // state to restore: directors (with ghosts), per-replica state, sweep counter, series length
  float *save = nullptr;
  CK(cudaMalloc(&save, (size_t)e->dir_floats * sizeof(float)));
  const int cur0 = e->cur, series0 = e->series_len;
  const bool graphs0 = e->use_graphs, prof0 = e->profile;
  std::vector<RepState> st(e->n_rep);
  unsigned long long sweep0 = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  auto done = [&](int code) {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    cudaFree(save);
    e->use_graphs = graphs0;
    e->profile = prof0;
    return code;
  };
#define CKT(call)                                                     \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) return done(cuda_fail(e_, #call));         \
  } while (0)
  CKT(cudaMemcpyAsync(save, e->d_dir[cur0], (size_t)e->dir_floats * sizeof(float), cudaMemcpyDeviceToDevice,
                      e->stream));
  CKT(cudaMemcpyAsync(st.data(), e->d_state, e->n_rep * sizeof(RepState), cudaMemcpyDeviceToHost, e->stream));
  CKT(cudaMemcpyAsync(&sweep0, e->d_sweep, sizeof sweep0, cudaMemcpyDeviceToHost, e->stream));
  CKT(cudaStreamSynchronize(e->stream));
  // the candidate plan decides whether a second buffer exists: the state always goes back into buffer 0
  auto restore = [&]() -> int {
    e->cur = 0;
    CK(cudaMemcpyAsync(e->d_dir[0], save, (size_t)e->dir_floats * sizeof(float), cudaMemcpyDeviceToDevice,
                       e->stream));
    CK(cudaMemcpyAsync(e->d_state, st.data(), e->n_rep * sizeof(RepState), cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(e->d_sweep, &sweep0, sizeof sweep0, cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(e->d_series_len, &series0, sizeof series0, cudaMemcpyHostToDevice, e->stream));
    e->series_len = series0;
    e->ghosts_dirty = false;  // the saved buffer carries its ghost cells
    CK(cudaStreamSynchronize(e->stream));
    return MCL_OK;
  };
  drop_graphs(e);
  e->use_graphs = false;
  e->profile = false;
  CKT(cudaEventCreate(&ev0));
  CKT(cudaEventCreate(&ev1));
  int cfg0 = 0, seg0 = 0;
  if ((rc = fused_get_cfg(e, &cfg0, nullptr, &seg0, nullptr))) return done(rc);
  std::vector<std::pair<int, int>> cand;
  fused_plan_candidates(e, cand);
  if (std::find(cand.begin(), cand.end(), std::make_pair(cfg0, seg0)) == cand.end()) cand.push_back({cfg0, seg0});
  double best = 1e300, t_default = 0;
  std::pair<int, int> pick{cfg0, seg0};
  for (const auto &c : cand) {
    if ((rc = fused_set_plan(e, c.first, c.second))) return done(rc);
    if ((rc = mcl_sweeps(e, 1, 1))) return done(rc);  // warm-up
    CKT(cudaEventRecord(ev0, e->stream));
    if ((rc = mcl_sweeps(e, trial_sweeps, 1))) return done(rc);
    CKT(cudaEventRecord(ev1, e->stream));
    CKT(cudaEventSynchronize(ev1));
    float ms = 0.f;
    CKT(cudaEventElapsedTime(&ms, ev0, ev1));
    const double per = ms / trial_sweeps;
    if (c.first == cfg0 && c.second == seg0) t_default = per;
    if (per < best) {
      best = per;
      pick = c;
    }
    if ((rc = restore())) return done(rc);
    if ((rc = fused_check_error(e))) return done(rc);
  }
  if ((rc = fused_set_plan(e, pick.first, pick.second))) return done(rc);
  if (out) {
    int ty = 0, seg = 0, items = 0;
    fused_get_cfg(e, nullptr, &ty, &seg, &items);
    out->tile_config = pick.first;
    out->rows_per_tile = ty;
    out->threads_per_cta = fused_threads(pick.first);
    out->planes_per_segment = seg;
    out->work_items = items;
    out->candidates = (int)cand.size();
    out->ms_per_sweep = best;
    out->ms_default = t_default;
  }
#undef CKT
  return done(MCL_OK);
}

int mcl_set_plan(mcl_engine *e, int tile_config, int planes_per_segment) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (!e->fused) return fail(MCL_ERR_STATE, "mcl_set_plan: the engine does not run the tiled sweep");
  drop_graphs(e);
  return fused_set_plan(e, tile_config, planes_per_segment);
}

int mcl_get_plan(mcl_engine *e, mcl_tuning *out) {
  if (!e || !out) return fail(MCL_ERR_ARG, "null argument");
  if (!e->fused) return fail(MCL_ERR_STATE, "mcl_get_plan: the engine does not run the tiled sweep");
  int cfg = 0, ty = 0, seg = 0, items = 0;
  const int rc = fused_get_cfg(e, &cfg, &ty, &seg, &items);
  if (rc) return rc;
  *out = mcl_tuning{};
  out->tile_config = cfg;
  out->rows_per_tile = ty;
  out->threads_per_cta = fused_threads(cfg);
  out->planes_per_segment = seg;
  out->work_items = items;
  return MCL_OK;
}

// ---- z-slab decomposition of one lattice over several processes ------------------------------------------------
int mcl_zslab_init(mcl_engine *e, int nz_global, int z_offset, int periodic_z, long long *plane_floats) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (e->zslab) return fail(MCL_ERR_STATE, "mcl_zslab_init: already a z-slab engine");
  if (!e->fused || e->n_rep != 1 || e->d_mlp || e->record_dec)
    return fail(MCL_ERR_STATE, "mcl_zslab_init: needs a bulk or slab engine of one replica on the tiled sweep, without a "
                               "learned proposal or decision recording");
  RepDesc &D = e->desc[0];
  if (D.periodic[2]) return fail(MCL_ERR_ARG, "mcl_zslab_init: create the local replica with a free z axis; the global "
                                              "z boundary is periodic_z");
  if (D.nz < 3) return fail(MCL_ERR_ARG, "mcl_zslab_init: the local replica needs at least one owned plane and two halos");
  if (z_offset < 0 || nz_global < 1 || z_offset + D.nz - 2 > nz_global)
    return fail(MCL_ERR_ARG, "mcl_zslab_init: owned planes %d..%d outside the global 0..%d", z_offset,
                z_offset + D.nz - 3, nz_global - 1);
  if (periodic_z && e->geo == GEO_SLAB) return fail(MCL_ERR_ARG, "mcl_zslab_init: the slab geometry has a free z axis");
  if (periodic_z && nz_global % 2)
    return fail(MCL_ERR_INPUT, "mcl_zslab_init: a periodic z axis needs an even number of planes (%d)", nz_global);
  CK(cudaStreamSynchronize(e->stream));
  int cfg = 0, seg = 0;
  int rc = fused_get_cfg(e, &cfg, nullptr, &seg, nullptr);
  if (rc) return rc;
  D.zslab = 1;
  D.zoff = z_offset - 1;
  D.nzg = nz_global;
  D.periodic[2] = periodic_z ? 1 : 0;
  D.n_valid = (double)D.nx * D.ny * nz_global;
  CK(cudaMemcpy(e->d_desc, &D, sizeof D, cudaMemcpyHostToDevice));
  e->zslab = true;
  drop_graphs(e);
  const bool flip = e->model.flip != 0 || e->model.potential == POT_PEAR;
  if ((rc = fused_set_plan(e, fused_is_pass_plan(e) ? cfg : (flip ? 4 : 2), 0))) return rc;
  if (plane_floats) *plane_floats = 3ll * D.py * D.px;
  return MCL_OK;
}

int mcl_zslab_pack(mcl_engine *e, float *send_lo, float *send_hi) {
  if (!e || !e->zslab) return fail(MCL_ERR_STATE, "mcl_zslab_pack: not a z-slab engine");
  int rc = refresh_ghosts(e);  // the planes go out whole, ghost cells included
  if (rc) return rc;
  CK(launch_zslab_planes(e->ctx(), e->d_dir[e->cur], send_lo, send_hi, 1));
  e->launches++;
  return MCL_OK;
}

int mcl_zslab_unpack(mcl_engine *e, const float *recv_lo, const float *recv_hi) {
  if (!e || !e->zslab) return fail(MCL_ERR_STATE, "mcl_zslab_unpack: not a z-slab engine");
  CK(launch_zslab_planes(e->ctx(), e->d_dir[e->cur], const_cast<float *>(recv_lo), const_cast<float *>(recv_hi), 0));
  e->launches++;
  return MCL_OK;
}

int mcl_zslab_pass(mcl_engine *e, int colour, int measure) {
  if (!e || !e->zslab) return fail(MCL_ERR_STATE, "mcl_zslab_pass: not a z-slab engine");
  if (colour != 0 && colour != 1) return fail(MCL_ERR_ARG, "mcl_zslab_pass: colour must be 0 or 1");
  int rc = refresh_ghosts(e);
  if (rc) return rc;
  return fused_pass(e, colour, measure != 0);
}

int mcl_zslab_sums(mcl_engine *e, int measure, double *d_sums) {
  if (!e || !e->zslab) return fail(MCL_ERR_STATE, "mcl_zslab_sums: not a z-slab engine");
  if (!d_sums) return fail(MCL_ERR_ARG, "mcl_zslab_sums: null buffer");
  return fused_item_sums(e, measure ? 1 : 0, d_sums);
}

int mcl_zslab_finalize(mcl_engine *e, const double *d_sums, int measure) {
  if (!e || !e->zslab) return fail(MCL_ERR_STATE, "mcl_zslab_finalize: not a z-slab engine");
  if (!d_sums) return fail(MCL_ERR_ARG, "mcl_zslab_finalize: null sums");
  int rc;
  if (measure && (rc = ensure_series(e, e->series_len + 1))) return rc;
  if ((rc = fused_finalize_global(e, d_sums, measure ? 1 : 0))) return rc;
  if (measure) e->series_len++;
  return MCL_OK;
}

int mcl_record_decisions(mcl_engine *e, int enable) {
  if (!e) return fail(MCL_ERR_ARG, "null engine");
  if (enable && !e->d_dec) {
    CK(cudaMalloc(&e->d_dec, (size_t)e->n_sites));
    CK(cudaMemsetAsync(e->d_dec, 0, (size_t)e->n_sites, e->stream));
  }
  e->record_dec = enable != 0;
  return MCL_OK;
}

int mcl_read_decisions(mcl_engine *e, int replica, unsigned char *out) {
  int rc = check_rep(e, replica, false);
  if (rc) return rc;
  if (!e->d_dec) return fail(MCL_ERR_STATE, "decision recording was never enabled");
  if (!out) return fail(MCL_ERR_ARG, "null output");
  const RepDesc &D = e->desc[replica];
  CK(cudaMemcpyAsync(out, e->d_dec + D.site_off, (size_t)D.nx * D.ny * D.nz, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return MCL_OK;
}

}  // extern "C"
