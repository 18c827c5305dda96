// Tiled sweeps on TMA-streamed planes, host side (tensor maps, work items, tile configuration, launches): the fused
// two-colour kernel (sweep_fused.cuh) and the in-place colour passes (sweep_pass.cuh) share the work items, the
// per-item partials and the finalisation; the tile configuration selects the kernel.
#include <stdlib.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "fused.h"
#include "sweep_pass.cuh"

namespace mcl {

// 0, 1: fused (7 slots of TY + 4 rows: one CTA per SM either way); 2-4: colour passes (4 slots of TY + 2 rows; 3 has
// 2 CTAs per SM, for flip models; 4 has 32-wide tiles, for lattices whose width is not a multiple of 64).
static const FusedCfg kCfgs[kNumCfgs] = {{14, 256, 1, 0, 64}, {28, 512, 1, 0, 64}, {16, 256, 3, 1, 64},
                                         {16, 256, 2, 1, 64}, {16, 128, 5, 1, 32}};

struct FusedPlan {
  int cfg = 0, tx = 64, ty = 14, seg = 32;
  FusedCfg C{};              // the tile configuration (kCfgs[cfg], or the learned plan's own)
  bool learned = false;      // the learned colour passes' plan: its kernel sets its own shared-memory limit
  FusedPlan *lplan = nullptr;  // that plan, built at the first learned sweep
  int seg_override = 0;  // planes per z segment chosen by the autotuner (0: heuristic)
  int n_items = 0;
  FusedItem *d_items = nullptr;
  CUtensorMap *d_tmaps = nullptr;
  double *d_partials = nullptr;
  int *d_first = nullptr;  // first item of each replica (n_rep + 1)
  unsigned int *d_err = nullptr;
  size_t smem = 0;
  long long timeout_ns = 2000000000ll;
  int skip_first_load = 0;
};

// ---- host side ----------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

bool fused_supported(const mcl_engine *e) {
  if (e->geo != GEO_BULK && e->geo != GEO_SLAB) return false;
  return get_encode() != nullptr;
}

// Box of `cells` half-row cells (TX / 2 + 8) and `rows` padded rows (fused: TY + 4, colour pass: TY + 2).
static int encode_map(CUtensorMap *map, float *base, const RepDesc &D, int cells, int rows) {
  // 5-D view of the split layout: (half-row cell, x parity, padded row, plane, component)
  cuuint64_t dims[5] = {(cuuint64_t)D.hp, 2, (cuuint64_t)D.py, (cuuint64_t)D.nz, 3};
  cuuint64_t strides[4] = {(cuuint64_t)D.hp * 4, (cuuint64_t)D.px * 4, (cuuint64_t)D.px * D.py * 4, (cuuint64_t)D.comp * 4};
  cuuint32_t box[5] = {(cuuint32_t)cells, 2, (cuuint32_t)rows, 1, 3};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = get_encode()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base + D.off, dims, strides, box, es,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MCL_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return MCL_OK;
}

#define CKF(call)                                        \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Tile and segment choice for configuration `cfg`: z segments sized so that the number of work items is close to
// a multiple of the resident CTAs, with segments long enough that the extra planes of each stay cheap (fused: four
// loaded, two of them computed; colour pass: two loaded).
static void choose_segments(const mcl_engine *e, FusedPlan &P, int sms) {
  const FusedCfg &C = P.C;
  P.tx = C.tx;
  P.ty = C.ty;
  long long tiles = 0, maxz = 1;
  for (auto &D : e->desc) {
    tiles += (long long)((D.nx + P.tx - 1) / P.tx) * ((D.ny + P.ty - 1) / P.ty);
    maxz = std::max<long long>(maxz, D.nz);
  }
  const long long slots = (long long)C.ctas_per_sm * sms;
  int best = 1;
  double best_score = -1;
  for (int nseg = 1; nseg <= 256; nseg++) {
    const double seg_len = (double)maxz / nseg;
    if (seg_len < 6 && nseg > 1) break;
    const long long items = tiles * nseg;
    const double waves = (double)items / slots;
    const double eff = waves / std::ceil(waves);
    const double extra = C.kind ? 2.0 * 0.15 : 4.0 * 0.35;  // extra planes mostly hit L2
    const double score = eff * seg_len / (seg_len + extra);
    if (score > best_score + 1e-9) {
      best_score = score;
      best = nseg;
    }
  }
  P.seg = (int)((maxz + best - 1) / best);
  if (P.seg_override > 0) P.seg = (int)std::min<long long>(P.seg_override, maxz);
}

static int choose_cfg(const mcl_engine *e) {
  // Colour passes (faster than the fused kernel on every measured workload): 3 CTAs per SM fit the 80 registers
  // of the non-flip kernels; flip models (a second trial per site) need the 2-CTA variant's registers.
  const char *env = getenv("MCL_FUSED_CFG");
  if (env) return std::max(0, std::min(kNumCfgs - 1, atoi(env)));
  const bool flip = e->model.flip != 0 || e->model.potential == POT_PEAR;
  return flip ? 3 : 2;
}

static int prepare_kernel(mcl_engine *e, FusedPlan *P);
static void free_plan(FusedPlan *P);

// The fused plans read one director buffer and write the other; the colour passes and the learned passes update
// one buffer in place. The second buffer (211 MB for a 256^3 lattice) therefore exists only while a fused plan is
// selected: switching to an in-place plan brings the state into buffer 0 and frees buffer 1. The learned plan's
// tensor maps name the buffers, so it is rebuilt at the next learned sweep.
static int set_buffers(mcl_engine *e, FusedPlan *P) {
  const bool two = P->C.kind == 0;
  if (two == (e->d_dir[1] != nullptr)) return MCL_OK;
  CKF(cudaStreamSynchronize(e->stream));
  if (two) {
    CKF(cudaMalloc(&e->d_dir[1], (size_t)e->dir_floats * sizeof(float)));
    CKF(cudaMemsetAsync(e->d_dir[1], 0, (size_t)e->dir_floats * sizeof(float), e->stream));
  } else {
    if (e->cur == 1)
      CKF(cudaMemcpyAsync(e->d_dir[0], e->d_dir[1], (size_t)e->dir_floats * sizeof(float), cudaMemcpyDeviceToDevice,
                          e->stream));
    CKF(cudaStreamSynchronize(e->stream));
    CKF(cudaFree(e->d_dir[1]));
    e->d_dir[1] = nullptr;
    e->cur = 0;
  }
  if (P->lplan) {
    free_plan(P->lplan);
    delete P->lplan;
    P->lplan = nullptr;
  }
  return MCL_OK;
}

static int build_items(mcl_engine *e, FusedPlan *P) {
  if (!P->learned) {
    P->C = kCfgs[P->cfg];
    const int rc = set_buffers(e, P);
    if (rc) return rc;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  choose_segments(e, *P, sms);
  // maps of buffer 0 and buffer 1 per replica (buffer 0's twice while there is one buffer: the state is in buffer 0)
  std::vector<CUtensorMap> maps(2 * e->n_rep);
  for (int r = 0; r < e->n_rep; r++)
    for (int b = 0; b < 2; b++) {
      int rc = encode_map(&maps[2 * r + b], e->d_dir[e->d_dir[1] ? b : 0], e->desc[r], P->tx / 2 + 8,
                          P->ty + (P->C.kind ? 2 : 4));
      if (rc) return rc;
    }
  cudaFree(P->d_tmaps);
  cudaFree(P->d_items);
  cudaFree(P->d_first);
  cudaFree(P->d_partials);
  CKF(cudaMalloc(&P->d_tmaps, maps.size() * sizeof(CUtensorMap)));
  CKF(cudaMemcpy(P->d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  std::vector<FusedItem> items;
  std::vector<int> first;
  for (int r = 0; r < e->n_rep; r++) {
    first.push_back((int)items.size());
    const RepDesc &D = e->desc[r];
    const int zlo = D.zslab ? 1 : 0, zhi = D.zslab ? D.nz - 1 : D.nz;  // a z-slab's halo planes are not swept
    for (int z0 = zlo; z0 < zhi; z0 += P->seg)
      for (int y0 = 0; y0 < D.ny; y0 += P->ty)
        for (int x0 = 0; x0 < D.nx; x0 += P->tx) items.push_back(FusedItem{r, x0, y0, z0, std::min(zhi, z0 + P->seg)});
  }
  first.push_back((int)items.size());
  P->n_items = (int)items.size();
  CKF(cudaMalloc(&P->d_items, items.size() * sizeof(FusedItem)));
  CKF(cudaMemcpy(P->d_items, items.data(), items.size() * sizeof(FusedItem), cudaMemcpyHostToDevice));
  CKF(cudaMalloc(&P->d_first, first.size() * sizeof(int)));
  CKF(cudaMemcpy(P->d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice));
  CKF(cudaMalloc(&P->d_partials, (size_t)P->n_items * kPartials * sizeof(double)));
  const bool pass = P->C.kind == 1;
  const int nsl = pass ? NSLP : NSL;
  const size_t slot_floats = ((size_t)3 * (P->tx + 16) * (P->ty + (pass ? 2 : 4)) + 31) / 32 * 32;
  P->smem = 128 + (size_t)nsl * slot_floats * sizeof(float) + nsl * sizeof(unsigned long long);
  return P->learned ? MCL_OK : prepare_kernel(e, P);
}

int fused_create(mcl_engine *e) {
  FusedPlan *P = new FusedPlan();
  e->fused = P;
  P->cfg = choose_cfg(e);
  CKF(cudaMalloc(&P->d_err, sizeof(unsigned int)));
  CKF(cudaMemset(P->d_err, 0, sizeof(unsigned int)));
  return build_items(e, P);
}

// Selects a plan and rebuilds the work items, tensor maps and buffers for it; if that fails (an allocation), the
// previous plan is rebuilt, so the engine keeps a consistent plan, and the first error is returned.
static int apply_plan(mcl_engine *e, int cfg, int seg) {
  FusedPlan *P = e->fused;
  const int cfg0 = P->cfg, seg0 = P->seg_override;
  P->cfg = cfg;
  P->seg_override = seg;
  const int rc = build_items(e, P);
  if (rc == MCL_OK) return MCL_OK;
  P->cfg = cfg0;
  P->seg_override = seg0;
  build_items(e, P);
  return rc;
}

int fused_set_cfg(mcl_engine *e, int cfg) {
  if (!e->fused) return fail(MCL_ERR_STATE, "this engine does not use the fused tiled sweep");
  if (cfg < 0 || cfg >= kNumCfgs) return fail(MCL_ERR_ARG, "tile configuration %d outside 0..%d", cfg, kNumCfgs - 1);
  CKF(cudaStreamSynchronize(e->stream));
  return apply_plan(e, cfg, e->fused->seg_override);
}

int fused_set_plan(mcl_engine *e, int cfg, int seg) {
  if (!e->fused) return fail(MCL_ERR_STATE, "this engine does not use the fused tiled sweep");
  if (cfg < 0 || cfg >= kNumCfgs) return fail(MCL_ERR_ARG, "tile configuration %d outside 0..%d", cfg, kNumCfgs - 1);
  if (kCfgs[cfg].kind == 0 && e->zslab)
    return fail(MCL_ERR_STATE, "a z-slab engine runs the colour passes (tile configurations 2-%d)", kNumCfgs - 1);
  CKF(cudaStreamSynchronize(e->stream));
  return apply_plan(e, cfg, std::max(0, seg));
}

void fused_plan_candidates(const mcl_engine *e, std::vector<std::pair<int, int>> &out) {
  out.clear();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  int maxz = 1;
  for (auto &D : e->desc) maxz = std::max(maxz, D.nz);
  for (int cfg = 0; cfg < kNumCfgs; cfg++) {
    FusedPlan P;
    P.cfg = cfg;
    P.C = kCfgs[cfg];
    choose_segments(e, P, sms);
    std::vector<int> segs = {P.seg, P.seg * 2, (P.seg + 1) / 2, maxz};
    // lattices too small to give every SM a work item (C1's 32^3: 10 items) also try short segments in the colour
    // passes, which trade two extra planes per item for more items in flight
    long long tiles = 0;
    for (auto &D : e->desc) tiles += (long long)((D.nx + P.tx - 1) / P.tx) * ((D.ny + P.ty - 1) / P.ty);
    const bool few = P.C.kind == 1 && tiles * ((maxz + P.seg - 1) / P.seg) < sms;
    if (few)
      for (int sg : {2, 3, 4}) segs.push_back(sg);
    std::sort(segs.begin(), segs.end());
    segs.erase(std::unique(segs.begin(), segs.end()), segs.end());
    for (int sg : segs)
      if (sg >= 6 || sg == maxz || (few && sg >= 2)) out.push_back({cfg, std::min(sg, maxz)});
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
}

int fused_threads(int cfg) { return kCfgs[std::max(0, std::min(kNumCfgs - 1, cfg))].nt; }

int fused_get_cfg(const mcl_engine *e, int *cfg, int *ty, int *seg, int *items) {
  if (!e->fused) return fail(MCL_ERR_STATE, "this engine does not use the fused tiled sweep");
  if (cfg) *cfg = e->fused->cfg;
  if (ty) *ty = e->fused->ty;
  if (seg) *seg = e->fused->seg;
  if (items) *items = e->fused->n_items;
  return MCL_OK;
}

static void free_plan(FusedPlan *P) {
  cudaFree(P->d_items);
  cudaFree(P->d_tmaps);
  cudaFree(P->d_partials);
  cudaFree(P->d_first);
}

int fused_learned_view(mcl_engine *e, LearnedPassView *v) {
  FusedPlan *P = e->fused;
  if (!P) return fail(MCL_ERR_STATE, "the learned colour passes need the tiled sweep");
  if (!P->lplan) {
    FusedPlan *L = new FusedPlan();
    L->learned = true;
    L->C = FusedCfg{8, 256, 2, 1, 64};  // 64 x 8 tiles: 256 sites of a colour per plane, one tcgen05 batch
    L->cfg = -1;
    const int rc = build_items(e, L);
    if (rc) {
      free_plan(L);
      delete L;
      return rc;
    }
    P->lplan = L;
  }
  v->tmaps = P->lplan->d_tmaps;
  v->items = P->lplan->d_items;
  v->n_items = P->lplan->n_items;
  v->partials = P->lplan->d_partials;
  v->first = P->lplan->d_first;
  return MCL_OK;
}

void fused_destroy(mcl_engine *e) {
  FusedPlan *P = e->fused;
  if (!P) return;
  if (P->lplan) {
    free_plan(P->lplan);
    delete P->lplan;
  }
  cudaFree(P->d_items);
  cudaFree(P->d_tmaps);
  cudaFree(P->d_partials);
  cudaFree(P->d_first);
  cudaFree(P->d_err);
  delete P;
  e->fused = nullptr;
}

static FusedLaunch launch_desc(const mcl_engine *e, const FusedPlan *P) {
  FusedLaunch l;
  l.geo = e->geo;
  l.cfg = P->cfg;
  l.flip = e->model.flip != 0 || e->model.potential == POT_PEAR;
  l.pxy = true;
  for (const auto &D : e->desc) l.pxy = l.pxy && D.periodic[0] && D.periodic[1];
  l.chiral = e->model.potential == POT_GHRL && e->model.sigma != 0.f;
  l.field = e->model.field_on != 0;
  l.n_items = P->n_items;
  l.smem = P->smem;
  l.stream = e->stream;
  return l;
}

static cudaError_t dispatch(const mcl_engine *e, const FusedArgs &a, const FusedLaunch &l) {
  if (kCfgs[l.cfg].kind == 1) {
    if (e->model.potential == POT_GHRL) return launch_pass_ghrl(e->model, a, l);
    if (e->model.potential == POT_PEAR) return launch_pass_pear(e->model, a, l);
    return launch_pass_ll(e->model, a, l);
  }
  if (e->model.potential == POT_GHRL) return launch_fused_ghrl(e->model, a, l);
  if (e->model.potential == POT_PEAR) return launch_fused_pear(e->model, a, l);
  return launch_fused_ll(e->model, a, l);
}

// Sets the dynamic shared-memory limit of the kernel this plan launches (once per plan, so that launches inside a
// stream capture make no attribute calls).
static int prepare_kernel(mcl_engine *e, FusedPlan *P) {
  FusedLaunch l = launch_desc(e, P);
  l.prepare = true;
  FusedArgs a{};
  const cudaError_t err = dispatch(e, a, l);
  if (err != cudaSuccess) return cuda_fail(err, "fused sweep: shared-memory attribute");
  return MCL_OK;
}

int fused_launches_per_sweep(const mcl_engine *e) { return e->fused && kCfgs[e->fused->cfg].kind == 1 ? 3 : 2; }

int fused_sweep(mcl_engine *e, bool measure, cudaEvent_t ev0, cudaEvent_t ev1) {
  FusedPlan *P = e->fused;
  const bool pass = kCfgs[P->cfg].kind == 1;
  FusedArgs a;
  a.tmaps = P->d_tmaps;
  a.out = e->d_dir[pass ? e->cur : e->cur ^ 1];  // colour passes update in place
  a.reps = e->d_desc;
  a.st = e->d_state;
  a.items = P->d_items;
  a.partials = P->d_partials;
  a.sweep_ctr = e->d_sweep;
  a.err = P->d_err;
  a.cur = e->cur;
  a.measure = measure ? 1 : 0;
  a.timeout_ns = P->timeout_ns;
  a.skip_first_load = P->skip_first_load;
  a.colour = 0;
  if (ev0) CKF(cudaEventRecord(ev0, e->stream));
  const FusedLaunch l = launch_desc(e, P);
  if (pass) {  // colour 0 without measurement, then colour 1 with the observables of the whole lattice
    FusedArgs a0 = a;
    a0.measure = 0;
    cudaError_t err = dispatch(e, a0, l);
    if (err != cudaSuccess) return cuda_fail(err, "colour pass launch");
    a.colour = 1;
    err = dispatch(e, a, l);
    if (err != cudaSuccess) return cuda_fail(err, "colour pass launch");
  } else {
    const cudaError_t err = dispatch(e, a, l);
    if (err != cudaSuccess) return cuda_fail(err, "fused sweep launch");
    e->cur ^= 1;
  }
  if (ev1) CKF(cudaEventRecord(ev1, e->stream));
  e->launches += fused_launches_per_sweep(e);
  BlockTable t;
  t.first = P->d_first;
  LaunchCtx c = e->ctx();
  CKF(launch_finalize(c, t, P->d_partials, measure ? 1 : 0, e->d_series, e->d_series_len, e->d_done));
  return MCL_OK;
}

bool fused_is_pass_plan(const mcl_engine *e) { return e->fused && kCfgs[e->fused->cfg].kind == 1; }

int fused_pass(mcl_engine *e, int colour, bool measure) {
  FusedPlan *P = e->fused;
  if (!P || kCfgs[P->cfg].kind != 1) return fail(MCL_ERR_STATE, "single colour passes need a colour-pass plan");
  FusedArgs a;
  a.tmaps = P->d_tmaps;
  a.out = e->d_dir[e->cur];
  a.reps = e->d_desc;
  a.st = e->d_state;
  a.items = P->d_items;
  a.partials = P->d_partials;
  a.sweep_ctr = e->d_sweep;
  a.err = P->d_err;
  a.cur = e->cur;
  a.measure = measure && colour == 1 ? 1 : 0;
  a.timeout_ns = P->timeout_ns;
  a.skip_first_load = P->skip_first_load;
  a.colour = colour;
  const cudaError_t err = dispatch(e, a, launch_desc(e, P));
  if (err != cudaSuccess) return cuda_fail(err, "colour pass launch");
  e->launches += 1;
  return MCL_OK;
}

int fused_item_sums(mcl_engine *e, int measure, double *d_sums) {
  FusedPlan *P = e->fused;
  if (!P) return fail(MCL_ERR_STATE, "this engine does not use the tiled sweep");
  BlockTable t;
  t.first = P->d_first;
  CKF(launch_item_sums(e->ctx(), t, P->d_partials, measure, d_sums));
  e->launches += 1;
  return MCL_OK;
}

int fused_finalize_global(mcl_engine *e, const double *d_sums, int measure) {
  FusedPlan *P = e->fused;
  if (!P) return fail(MCL_ERR_STATE, "this engine does not use the tiled sweep");
  BlockTable t;
  t.first = P->d_first;
  CKF(launch_finalize(e->ctx(), t, P->d_partials, measure, e->d_series, e->d_series_len, e->d_done, d_sums));
  e->launches += 1;
  return MCL_OK;
}

int fused_check_error(mcl_engine *e) {
  if (!e->fused) return MCL_OK;
  unsigned int v = 0;
  CKF(cudaMemcpyAsync(&v, e->fused->d_err, sizeof v, cudaMemcpyDeviceToHost, e->stream));
  CKF(cudaStreamSynchronize(e->stream));
  return fused_report_error(e, v);
}

unsigned int *fused_error_word(mcl_engine *e) { return e->fused ? e->fused->d_err : nullptr; }

int fused_report_error(mcl_engine *e, unsigned int v) {
  if (!v || !e->fused) return MCL_OK;
  unsigned int zero = 0;
  CKF(cudaMemcpy(e->fused->d_err, &zero, sizeof zero, cudaMemcpyHostToDevice));
  return fail(MCL_ERR_CUDA, "fused sweep: a TMA load did not complete within %.3f s (error word 0x%x)",
              e->fused->timeout_ns * 1e-9, v);
}

void fused_set_test_hooks(mcl_engine *e, long long timeout_ns, int skip_first_load) {
  if (!e->fused) return;
  if (timeout_ns > 0) e->fused->timeout_ns = timeout_ns;
  e->fused->skip_first_load = skip_first_load;
}

}  // namespace mcl
