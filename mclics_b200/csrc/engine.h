// Engine internals shared by the C-ABI implementation (engine.cpp), the fused kernel launcher and the driver.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/mclics_b200.h"
#include "common.cuh"
#include "launch.h"

namespace mcl {

// Sets the thread's last error message and returns code.
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t err, const char *what);

struct FusedPlan;  // fused tiled sweep (sweep_fused.cu)
struct MlpDev;     // learned proposal weights in device layout (learned.cu)
struct MlpTC;      // the same in the tcgen05 layout (mlp_tc.cuh)
int learned_check_error(mcl_engine *e);
// A learned-sweep error word read by the caller: non-zero is cleared and turned into MCL_ERR_CUDA.
int learned_report_error(mcl_engine *e, unsigned word);

}  // namespace mcl

struct mcl_engine {
  mcl_model model_in;
  mcl::ModelDev model;
  int schedule = MCL_SCHED_CHECKER2;
  int geo = mcl::GEO_BULK;
  int n_rep = 0;
  std::vector<mcl_replica> rep_in;
  std::vector<mcl::RepDesc> desc;  // host copy of the layouts
  long long dir_floats = 0;        // floats per director buffer
  long long n_sites = 0;           // total sites over all replicas
  long long max_sites = 0;         // largest replica

  cudaStream_t stream = nullptr;
  int device = 0;
  mcl::RepDesc *d_desc = nullptr;
  mcl::RepState *d_state = nullptr;
  float *d_dir[2] = {nullptr, nullptr};
  int cur = 0;  // which director buffer holds the current state
  uint8_t *d_pt = nullptr;
  float *d_nrm = nullptr;
  float *d_stage = nullptr;  // AoS staging for upload/download (max_sites * 3 floats)
  unsigned long long *d_sweep = nullptr;
  unsigned int *d_done = nullptr;
  int *d_series_len = nullptr;
  mcl::ObsRecord *d_series = nullptr;
  int series_cap = 0;  // rows
  int series_len = 0;  // host mirror
  mcl::ObsRecord *d_probe = nullptr;
  int *d_probe_len = nullptr;  // unused length slot for probe records
  double *d_partials = nullptr;
  uint8_t *d_dec = nullptr;
  bool record_dec = false;
  bool ghosts_dirty = true;
  bool geometry_set = true;

  mcl::BlockTable half, boxes, sites;
  std::vector<int> host_pt;  // point types (GEO_PT), for n_valid
  mcl::FusedPlan *fused = nullptr;
  cudaStream_t own_stream = nullptr;
  bool profile = false;
  bool zslab = false;  // replica 0 is a z-slab of a larger lattice (mcl_zslab_init): pass-level API only
  std::vector<cudaEvent_t> ev_pool;  // pairs (start, stop) of timed sweeps
  size_t ev_used = 0;
  double prof_ms = 0;          // time of already-read event pairs
  long long prof_sweeps = 0;
  long long launches = 0;      // kernels launched by this engine
  mcl::MlpDev *d_mlp = nullptr;  // learned proposal (null: plain proposal)
  mcl::MlpTC *d_mlp_tc = nullptr;  // the same weights in the tcgen05 layout
  unsigned *d_lerr = nullptr;      // learned-sweep error word
  bool mlp_tc = true;              // learned sweeps run the network on tcgen05
  bool learned_pass = true;        // ... as colour passes on streamed planes (bulk/slab with the tiled sweep)
  double *d_xpart = nullptr;   // scratch of mcl_measure_extras (allocated at its first call)
  float kappa_max = 500.f;
  bool adapt = true;           // ang_var adaptation after each sweep (the reference's behaviour)
  int mix_period = 1;          // with a learned proposal: every mix_period-th sweep learned, the others plain
  int mix_phase = 0;           // sweeps since the last learned one (mcl_set_proposal_mix)
  bool use_graphs = false;     // fused sweeps replayed from captured CUDA graphs (one or two sweeps each)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [measure]: the sweeps of one replay, from buffer graph_cur
  int graph_cur[2] = {0, 0};
  const void *graph_series = nullptr;             // series buffer the measuring graph writes
  cudaGraphExec_t graph_io = nullptr;  // mcl_sweeps_io's step (input kernel, one measured sweep, output kernel)
  const void *graph_io_series = nullptr, *graph_io_stage = nullptr;  // the buffers it was captured with
  void *h_io = nullptr;      // mapped pinned staging of mcl_sweeps_io: error words, temperatures, observables records
  void *d_io = nullptr;      // its device address
  size_t h_io_bytes = 0;
  bool io_inflight = false;  // copies that read or write h_io may still be queued (an error return before the sync)

  mcl::LaunchCtx ctx() const {
    mcl::LaunchCtx c;
    c.model = model;
    c.n_replicas = n_rep;
    c.reps = d_desc;
    c.state = d_state;
    c.dir = d_dir[cur];
    c.pt = d_pt;
    c.nrm = d_nrm;
    c.sweep_ctr = d_sweep;
    c.decisions = record_dec ? d_dec : nullptr;
    c.stream = stream;
    c.adapt = (adapt && !d_mlp) ? 1 : 0;
    return c;
  }
};
