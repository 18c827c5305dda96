// Host-side launchers of the device kernels (implemented in the .cu files, used by engine.cpp).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace mcl {

struct FusedItem;

// Block work table: block b of a launch works on replica rep[b], items [base[b], base[b] + blockDim).
struct BlockTable {
  int n_blocks = 0;
  int *rep = nullptr;         // device
  long long *base = nullptr;  // device
  int *first = nullptr;       // device, n_replicas + 1 entries: first block of each replica
};

struct LaunchCtx {
  ModelDev model;
  int n_replicas;
  const RepDesc *reps;      // device
  RepState *state;          // device
  float *dir;               // device director buffer (current)
  const uint8_t *pt;        // device point types (GEO_PT replicas), may be null
  const float *nrm;         // device normals (GEO_PT replicas), may be null
  unsigned long long *sweep_ctr;  // device
  uint8_t *decisions;       // device, null unless recording
  cudaStream_t stream;
  int adapt = 1;            // ang_var adaptation after each sweep (off: the amplitude stays fixed)
};

constexpr int kThreads = 256;

// One sweep with the two-colour schedule, one thread per site and colour (in place).
cudaError_t launch_sweep_checker2_simple(const LaunchCtx &c, int geo, const BlockTable &half);
// One sweep in the reference CPU order (8 sublattices, i fastest) with the reference arithmetic (in place).
cudaError_t launch_sweep_ref8(const LaunchCtx &c, int geo, const BlockTable &boxes);
// Observables of the current state into partials[block][kPartials].
cudaError_t launch_observe(const LaunchCtx &c, int geo, const BlockTable &sites, double *partials);
// Boundary planes of a z-slab to (pack = 1: owned planes 1, nz - 2) or from (pack = 0: halo planes 0, nz - 1) the
// caller's buffers of 3 py px floats each; a null buffer skips its side.
cudaError_t launch_zslab_planes(const LaunchCtx &c, float *dir, float *lo, float *hi, int pack);
// mcl_sweeps_io's step input (temperatures from mapped host memory into the replicas' state) and output (series rows
// first_row .. first_row + n_rows - 1, or with series_len the newest n_rows, and the error words, null for absent
// ones, into mapped host memory).
cudaError_t launch_io_in(cudaStream_t stream, RepState *st, const float *host_T, int n_rep);
cudaError_t launch_io_out(cudaStream_t stream, const ObsRecord *series, long long first_row, const int *series_len,
                          int n_rows, int n_rep, ObsRecord *host_rec, const unsigned *err0, const unsigned *err1,
                          unsigned *host_words);
// Per-replica sums of the partials over a block table and the accepted rotations (kZslabSums doubles each).
cudaError_t launch_item_sums(const LaunchCtx &c, const BlockTable &items, const double *partials, int measure,
                             double *out);
// Per-replica reduction of the partials, S by Jacobi, ang_var adaptation, series record, counter advance; with
// gsums, from sums already reduced over z-slab processes instead of the local partials and acceptance counter.
cudaError_t launch_finalize(const LaunchCtx &c, const BlockTable &sites, const double *partials, int measure,
                            ObsRecord *series, int *series_len, unsigned int *done_ctr,
                            const double *gsums = nullptr);
// Periodic ghost cells (x then y) of every replica.
cudaError_t launch_refresh_ghosts(const LaunchCtx &c, int max_ny_nz, int max_px_nz);
// One sweep with the learned proposal (two colours, in place); mlp: weights in device layout (learned.cu). With
// measure, the observables of the final state go to partials[block of `half`][kPartials] (reduce them with
// launch_finalize over the same table).
struct MlpDev;
struct MlpTC;
struct LearnedMlp {
  const MlpDev *warp;  // weights for the mma.sync warps
  const MlpTC *tc;     // weights for tcgen05
  unsigned *err;       // error word (tensor-core timeout)
  bool use_tc;
};
// The learned sweep as two in-place colour passes on TMA-streamed planes (bulk and slab, tcgen05 network): the
// work items, tensor maps and per-item partials of a 64 x 8-tile plan (fused_learned_view); finalise with
// launch_finalize over `first` and `partials`.
struct LearnedPassView {
  const CUtensorMap *tmaps = nullptr;
  const FusedItem *items = nullptr;
  int n_items = 0;
  double *partials = nullptr;
  int *first = nullptr;
};
cudaError_t launch_learned_pass(const LaunchCtx &c, int geo, const LearnedPassView &v, const LearnedMlp &mlp,
                                float kappa_max, int measure, float *dir, int cur);
cudaError_t launch_sweep_learned(const LaunchCtx &c, int geo, const BlockTable &half, const LearnedMlp &mlp,
                                 float kappa_max, int measure, double *partials);
// AoS (reference layout) <-> padded SoA for one replica.
cudaError_t launch_unpack(const LaunchCtx &c, int replica, const RepDesc &host_desc, const float *aos);
cudaError_t launch_pack(const LaunchCtx &c, int replica, const RepDesc &host_desc, float *aos);
// Random initial directors of one replica (common.cuh random_director, Philox stream 2 keyed by `seed`).
cudaError_t launch_random_ic(const LaunchCtx &c, const RepDesc &host_desc, unsigned long long seed);

}  // namespace mcl
