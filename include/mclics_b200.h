/* mclics_b200 — B200-native checkerboard Metropolis sweep for McLics (C ABI).
 *
 * The reference exposes its GPU path as C++ classes: `class EvolveNGPU : public Evolve` with the constructor
 * (float *ni, int *pt, Parameters *params) (include/evolve.cuh:22-42), the four mode subclasses
 * {thermal,step,quench,electric}EvolveNGPU (include/evolve.cuh:43-67), selected by name in
 * src/simulator.cpp:45-53, whose run() loops (src/evolve_{thermal,step,quench,electric}.cu) call
 * Monte_Carlo_Step_GPU (src/evolve.cu:317-440) and energy_calculator_GPU (src/evolve.cu:442-478). This header
 * is the plain-C replacement for that boundary: POD structs instead of Parameters (include/parameters.h:18-98),
 * an opaque engine handle instead of the class with function-local statics (so many simulations, and batches of
 * replicas, live in one process), and an int status on every call instead of printf + exit(20).
 *
 * Every function returns MCL_OK (0) or an MCL_ERR_* code; mcl_last_error() gives the message of the last failure
 * on the calling thread. No function exits the process or throws. All director arrays crossing this boundary use
 * the reference layout: 3 floats per site, site (i, j, k) at index i + Nx (j + Ny k) (include/define.h:9-19). */
#ifndef MCLICS_B200_H_
#define MCLICS_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

#define MCL_MAX_SURFACES 16

enum mcl_status {
  MCL_OK = 0,
  MCL_ERR_ARG = 1,         /* invalid argument (sizes, indices, null pointers, unsupported combination) */
  MCL_ERR_CUDA = 2,        /* a CUDA call failed (message has the CUDA error string) */
  MCL_ERR_NOMEM = 3,       /* device or host allocation failed */
  MCL_ERR_STATE = 4,       /* call not valid in the engine's current state */
  MCL_ERR_INPUT = 5,       /* input file or parameter error (same checks as src/io.cpp:381-475) */
  MCL_ERR_IO = 6,          /* file could not be read or written */
  MCL_ERR_NONFINITE = 7,   /* a director uploaded or produced is NaN/Inf or has zero length */
  MCL_ERR_NO_DEVICE = 8    /* no CUDA device, or not an sm_100 device */
};

/* Pair potential (src/potential.cpp:19-56, selected in src/simulator.cpp:234-250). */
enum mcl_potential { MCL_POT_LL = 0, MCL_POT_GHRL = 1, MCL_POT_PEAR = 2 };
/* Geometry (src/geometry_{bulk,slab,sphere,custom}.cpp). bulk and slab are analytic on the device (no
 * point-type array); sphere and custom take pt and normals through mcl_set_geometry. */
enum mcl_geometry { MCL_GEOM_BULK = 0, MCL_GEOM_SLAB = 1, MCL_GEOM_SPHERE = 2, MCL_GEOM_CUSTOM = 3 };
/* Surface anchoring (src/anchoring_*.cpp, names in src/geometry.cpp:78-107). */
enum mcl_anchoring {
  MCL_ANCH_HOMEOTROPIC = 0,
  MCL_ANCH_RP = 1,
  MCL_ANCH_RP_TANGENT = 2,
  MCL_ANCH_FG = 3,
  MCL_ANCH_HOMEOTROPIC_GHRL = 4,
  MCL_ANCH_RP_GHRL = 5,
  MCL_ANCH_FG_GHRL = 6
};
/* Update order within a sweep.
 *  MCL_SCHED_REF8      the reference CPU's 8 sublattices by parity of (i, j, k), visited with i fastest
 *                      (src/evolve.cpp:106-119), with the reference's float/double arithmetic. Used to replay
 *                      the reference decision by decision.
 *  MCL_SCHED_CHECKER2  two colours by parity of i+j+k (production): a different but equally valid Metropolis
 *                      chain. The fused tiled kernel is used where the geometry allows it.
 *  MCL_SCHED_CHECKER2_SIMPLE  two colours, one thread per site and colour, no tiling (baseline / fallback). */
enum mcl_schedule { MCL_SCHED_REF8 = 0, MCL_SCHED_CHECKER2 = 1, MCL_SCHED_CHECKER2_SIMPLE = 2 };

/* Model shared by every replica of an engine (the physics part of Parameters, include/parameters.h:18-98). */
typedef struct mcl_model {
  int potential;              /* mcl_potential */
  float A, B1, C;             /* couplings (A: LL and pear; B1, C: pear) */
  float ghrl_lambda, ghrl_mu, ghrl_nu, ghrl_rho, ghrl_sigma; /* GHRL coefficients (src/io.cpp:346-371) */
  float field_dir[3];         /* field direction, unit length (src/main.cpp:97-106 normalises it) */
  float elecA, elecP;         /* dielectric and dipolar couplings (src/potential.cpp:59-63) */
  int flip_move;              /* n -> -n trial after each rotation (src/main.cpp:88: pear or elecP != 0) */
  int n_surfaces;
  int anch_type[MCL_MAX_SURFACES];     /* mcl_anchoring of surface s (pt = s + 2) */
  float anch_W[MCL_MAX_SURFACES];      /* anchoring strength */
  float anch_theta[MCL_MAX_SURFACES];  /* easy axis polar angle, degrees (rp, rp_tangent, rp_ghrl) */
  float anch_phi[MCL_MAX_SURFACES];    /* easy axis azimuth, degrees */
} mcl_model;

/* One lattice (replica). Replicas of one engine may differ in size, temperature, field magnitude and seed. */
typedef struct mcl_replica {
  int nx, ny, nz;
  int geometry;               /* mcl_geometry; slab forces z free, sphere forces all axes free */
  int periodic[3];            /* per axis: 1 periodic, 0 free (src/potential.cpp:64-74); periodic needs even N */
  float T;                    /* temperature (params->T) */
  float elecE;                /* field magnitude (1 outside the electric mode) */
  float ang_var;              /* initial rotation amplitude; the reference starts every run at 0.5 */
  unsigned long long seed;    /* seed of this replica's Philox draws (part of every draw's counter) */
} mcl_replica;

/* Observables of one replica after one sweep (FP64 reductions over FP32 site terms). */
typedef struct mcl_observables {
  double energy;        /* mean site energy: bonds counted twice, anchoring and field once (src/evolve.cpp:33-75) */
  double q[6];          /* mean (3 n n - I)/2: xx, xy, xz, yy, yz, zz (src/parameter_order.cpp:40-71) */
  double S;             /* largest eigenvalue of q (src/parameter_order.cpp:19-37) */
  double director[3];   /* its eigenvector */
  double nsum[3];       /* sum of n over the non-empty sites */
  double n_valid;       /* number of non-empty sites */
  double acceptance;    /* accepted rotations / n_valid in that sweep (flips excluded, src/evolve.cpp:195) */
  double ang_var;       /* rotation amplitude after the sweep's adaptation (src/evolve.cpp:211-220) */
  double sweep;         /* global sweep index of the record */
} mcl_observables;

typedef struct mcl_engine mcl_engine;

/* Creates an engine on the current CUDA device holding n_replicas lattices. Directors start at (0, 0, 1). In place
 * of the EvolveNGPU constructor (include/evolve.cuh:22-42) and the device allocations and RNG set-up at the start
 * of its run() (src/evolve_thermal.cu:48-66); mcl_destroy releases what the reference never frees. */
int mcl_create(const mcl_model *model, const mcl_replica *replicas, int n_replicas, int schedule,
               mcl_engine **out);
int mcl_destroy(mcl_engine *e);

/* Point types (0 empty, 1 bulk, s+2 surface s) and outward normals (3 floats per site) of a sphere or custom
 * replica, in the reference layout (src/geometry_sphere.cpp:32-58, src/geometry_custom.cpp:70-163). */
int mcl_set_geometry(mcl_engine *e, int replica, const int *pt, const float *normals);

/* Host <-> device directors of one replica (3 floats per site, reference layout). Upload rejects NaN/Inf and
 * zero-length directors on non-empty sites with MCL_ERR_NONFINITE and leaves the device state unchanged. */
int mcl_upload_directors(mcl_engine *e, int replica, const float *ni);
int mcl_download_directors(mcl_engine *e, int replica, float *ni);

/* Random initial condition of one replica on the device (replaces the host loop of `ic random`,
 * src/ic.cpp:38-65): every non-empty site gets an isotropic unit vector from Philox stream 2 keyed by `seed`
 * (uniform point of a ball, projected onto the sphere; bit-identical to the same computation on the host), empty
 * sites of a sphere or custom replica (0, 0, 1). Call mcl_set_geometry first for those. */
int mcl_random_directors(mcl_engine *e, int replica, unsigned long long seed);

/* Per-replica parameters; replica = -1 applies to all. T is the temperature the mode loops copy to the device
 * (src/evolve_thermal.cu:80), elecE the field magnitude the electric mode sweeps (src/evolve_electric.cu:80-82),
 * ang_var the rotation amplitude Monte_Carlo_Step_GPU adapts (src/evolve.cu:302-313, starting at 0.5 per run,
 * src/evolve_thermal.cu:43). */
int mcl_set_temperature(mcl_engine *e, int replica, float T);
int mcl_set_field(mcl_engine *e, int replica, float elecE);
int mcl_set_ang_var(mcl_engine *e, int replica, float ang_var);
int mcl_get_ang_var(mcl_engine *e, int replica, float *ang_var);
/* Global sweep counter (the Philox counter of the next sweep). No counterpart: the reference advances per-box
 * XORWOW states instead (src/evolve.cu:35-41). */
int mcl_set_sweep_counter(mcl_engine *e, unsigned long long sweep);
int mcl_get_sweep_counter(mcl_engine *e, unsigned long long *sweep);

/* Runs n sweeps on every replica (Monte_Carlo_Step_GPU, src/evolve.cu:317-440, with ang_var adapted on the
 * device: no host synchronisation per sweep). With measure != 0 the observables after every sweep are appended
 * to the engine's series (energy_calculator_GPU + Q_tensor + eigen, done on the device). Asynchronous: returns
 * after enqueueing; errors of the device work surface at the next synchronising call. */
int mcl_sweeps(mcl_engine *e, int n, int measure);
/* One step of a caller's measurement loop in one call and one host synchronisation: T (n_replicas floats, or
 * null to keep the temperatures) goes up, n measured sweeps run as mcl_sweeps(e, n, 1), and their records come
 * down into out[s * n_replicas + r] (sweep s, replica r), together with the kernels' error words. Both directions
 * pass through the engine's mapped pinned staging, moved by two small kernels on the engine's stream. The same as mcl_set_temperature per replica, mcl_sweeps and mcl_read_series (the loop of
 * src/evolve_thermal.cu:78-106), without their separate round trips. */
int mcl_sweeps_io(mcl_engine *e, int n, const float *T, mcl_observables *out);
/* Number of records in the series; reading copies them to the host (synchronises). */
int mcl_series_length(mcl_engine *e, int *n);
int mcl_read_series(mcl_engine *e, int replica, int first, int count, mcl_observables *out);
int mcl_clear_series(mcl_engine *e);
/* Sizes the series for `rows` records per replica, so that the sweeps appending them neither reallocate it (an
 * allocation and a host synchronisation) nor capture their graphs again. No counterpart in the reference, which
 * keeps no series (its loops fold each record into running sums, src/evolve_thermal.cu:84-95). */
int mcl_reserve_series(mcl_engine *e, int rows);
/* Observables of the current state (synchronises). acceptance/ang_var fields refer to the last sweep. */
int mcl_measure(mcl_engine *e, int replica, mcl_observables *out);
int mcl_synchronize(mcl_engine *e);

/* Records one byte per site for the sweeps that follow (bit 0: rotation accepted, bit 1: flip accepted,
 * bit 7: site visited); mcl_read_decisions copies those of the last sweep. Test hook for the replay harness (no
 * counterpart in the reference). */
int mcl_record_decisions(mcl_engine *e, int enable);
int mcl_read_decisions(mcl_engine *e, int replica, unsigned char *out);

/* Work of this engine goes to `stream` (a cudaStream_t of the current device; NULL restores the engine's own
 * stream), so a caller can order it with its own work and time it with its own events. No counterpart (the
 * reference uses the default stream). */
int mcl_set_stream(mcl_engine *e, void *stream);
/* Kernel timing: with enable != 0 every following sweep records CUDA events around its sweep kernel(s) (not the
 * per-sweep finalisation); mcl_profile_read returns their total time in ms and the number of sweeps timed, and
 * the number of kernels this engine has launched since creation. No counterpart in the reference. */
int mcl_profile(mcl_engine *e, int enable);
int mcl_profile_read(mcl_engine *e, double *sweep_kernel_ms, long long *timed_sweeps, long long *kernel_launches);

/* Failure-detection test hook: every wait of the fused tiled sweep on a TMA copy gives up after timeout_ns
 * (> 0 to change; default 2 s) and the sweep then reports MCL_ERR_CUDA at the next synchronising call, with
 * the context still usable. With withhold_first_load != 0 each CTA leaves its first copy unissued, so that
 * wait runs out; 0 restores normal operation. MCL_ERR_STATE if the engine does not use the fused sweep. No
 * counterpart in the reference. */
int mcl_debug_wait_limit(mcl_engine *e, long long timeout_ns, int withhold_first_load);

/* Runs a whole McLics input file in the current directory, like the reference program with a *GPU evolution
 * mode (src/main.cpp:83-125): same input grammar and validation, writes ic.csv, po.dat and
 * director_field_*.csv. The mode may be given with or without the GPU suffix. */
int mcl_run_input_file(const char *path);

/* Extra order parameters of the current state of one replica, on the device (Polarization, Splay_magnitude,
 * Splay_divergence, Radial_order of src/parameter_order.cpp:129-245; the reference computes them on the host after
 * copying the lattice back, src/parameter_order.cpp:249-295). director: the Q-tensor director of the same state
 * (mcl_observables.director), for P = |d . sum n| / N_valid. Radial orders are about the grid centre
 * (Nx/2, Ny/2, Nz/2) and about the z axis through it, skipping sites within half a spacing. The first call allocates
 * scratch for the engine's largest replica. Synchronises. */
typedef struct mcl_extras {
  double P, dtheta, divn;
  double Sr_sph, Pr_sph;  /* about the centre */
  double Sr_cyl, Pr_cyl;  /* about the z axis */
} mcl_extras;
int mcl_measure_extras(mcl_engine *e, int replica, const double director[3], mcl_extras *out);
/* Local order parameter of every site of one replica, on the device (lattice_order_parameter,
 * src/parameter_order.cpp:75-127, written in every snapshot by print_n, src/io.cpp:59-89): the largest eigenvalue
 * of Q over the site and its existing non-empty neighbours; NaN on empty sites. S: host array of Nx Ny Nz floats in
 * the reference order. Synchronises. */
int mcl_local_order(mcl_engine *e, int replica, float *S);

/* ---- Batched sweeps: tuning and graph replay (no counterpart in the reference: it runs one lattice per process,
 * src/evolve.cu:317-440) ----------------------------------------------------------------------------------------
 * The replicas of an engine are swept together: every work item (replica, tile, z segment) of every replica is one
 * CTA of one launch. A plan is a tile configuration and a number of planes per z segment. Tile configurations:
 *   0: fused sweep (both colours in one launch, ping-pong buffers), 64 x 14 sites, 256 threads per CTA;
 *   1: fused sweep, 64 x 28 sites, 512 threads;
 *   2: two in-place colour passes per sweep, 64 x 16 sites, 256 threads, 3 CTAs per SM;
 *   3: colour passes, 64 x 16 sites, 256 threads, 2 CTAs per SM (flip models: two trials per site);
 *   4: colour passes, 32 x 16 sites, 128 threads, 5 CTAs per SM (narrow lattices waste less of a tile).
 * The fused configurations need a second director buffer, allocated while one of them is selected and freed when a
 * colour-pass configuration is selected again. Every configuration gives bit-identical directors. Candidate plans:
 * per configuration the heuristic segment length, its double, its half and the whole depth; lattices that give
 * fewer work items than SMs also 2-4 planes in the colour passes. mcl_autotune times each candidate plan for
 * trial_sweeps measured sweeps on the engine's own replicas, keeps the fastest and restores the directors,
 * per-replica state, sweep counter and series, so the run continues as if it had not been called. MCL_ERR_STATE
 * unless the engine runs the tiled sweep (bulk/slab, plain proposal, no decision recording). */
typedef struct mcl_tuning {
  int tile_config;        /* 0..4 as above */
  int rows_per_tile;
  int threads_per_cta;
  int planes_per_segment;
  int work_items;         /* CTAs per sweep */
  int candidates;         /* plans timed */
  double ms_per_sweep;    /* the chosen plan: one sweep + its measurement */
  double ms_default;      /* the plan in use before the call */
} mcl_tuning;
int mcl_autotune(mcl_engine *e, int trial_sweeps, mcl_tuning *out);
/* Applies a plan (e.g. one mcl_autotune chose earlier) without timing: planes_per_segment <= 0 lets the heuristic
 * choose. mcl_get_plan fills the plan fields of *out (tile_config .. work_items; the timing fields are 0). No
 * counterpart in the reference, whose launch shape is fixed (src/evolve.cu:335-339, 409-410). */
int mcl_set_plan(mcl_engine *e, int tile_config, int planes_per_segment);
int mcl_get_plan(mcl_engine *e, mcl_tuning *out);

/* ---- Z-slab decomposition: one lattice over several processes, one GPU each (no counterpart in the reference,
 * which sweeps one lattice in one process on one GPU, src/evolve.cu:317-440) --------------------------------------
 * A process owns the global planes z_offset .. z_offset + nz_own - 1 of a lattice of nz_global planes. Its engine
 * has one replica (bulk or slab geometry) created with nz = nz_own + 2 and a free z axis; local planes 0 and
 * nz - 1 are halo copies of the neighbouring processes' boundary planes, and periodic_z gives the global z
 * boundary. Site draws and slab surfaces use global plane indices, so the processes together take exactly the
 * decisions one engine sweeping the whole lattice takes. The engine runs the colour-pass kernel; the caller moves
 * the boundary planes between processes (e.g. NCCL send/recv over NVLink) and sums the observables. One sweep:
 *   for colour 0, 1: mcl_zslab_pass(colour); mcl_zslab_pack(send_lo, send_hi); exchange; mcl_zslab_unpack(...)
 *   mcl_zslab_sums(measure, sums); sum the sums over the processes; mcl_zslab_finalize(sums, measure)
 * where send_lo (the lowest owned plane) goes to the lower neighbour's recv_hi and send_hi to the upper neighbour's
 * recv_lo. Before the first sweep, pack, exchange and unpack once. Buffers are device memory the caller owns:
 * plane buffers of *plane_floats floats ([component][padded row][cell], ghost cells included), sums of 11 doubles
 * (energy, Q xx xy xz yy yz zz, sum n, accepted rotations). Every call is asynchronous on the engine's stream.
 * A z-slab engine refuses mcl_sweeps, mcl_measure and mcl_autotune; the directors it downloads are its nz_own + 2
 * local planes. */
int mcl_zslab_init(mcl_engine *e, int nz_global, int z_offset, int periodic_z, long long *plane_floats);
int mcl_zslab_pass(mcl_engine *e, int colour, int measure);
int mcl_zslab_pack(mcl_engine *e, float *send_lo, float *send_hi);          /* null: skip that side */
int mcl_zslab_unpack(mcl_engine *e, const float *recv_lo, const float *recv_hi); /* null: no neighbour there */
int mcl_zslab_sums(mcl_engine *e, int measure, double *d_sums);
int mcl_zslab_finalize(mcl_engine *e, const double *d_sums, int measure);
/* With enable != 0, mcl_sweeps (and mcl_sweeps_io) replay a captured CUDA graph of one sweep (colour-pass plans)
 * or two (the ping-pong fused plans 0 and 1), captured at the first call and again after the plan, the series buffer
 * or the test hooks change, instead of launching kernels one by one; results are identical. Profiling (mcl_profile)
 * uses direct launches. */
int mcl_set_graphs(mcl_engine *e, int enable);

/* ---- Learned Metropolis-Hastings proposal (no counterpart in the reference) ----------------------------------
 * Per site, a 7 -> 64 -> 64 -> 4 MLP with SiLU reads the neighbour Q-tensor sum sum_j (3 n_j n_j^T - I)/2 divided by
 * 6 (xx, xy, xz, yy, yz, zz) and T, and gives an axis mu (outputs 0..2, normalised) and a concentration
 * kappa = clip(softplus(output 3), 1e-3, kappa_max). The trial director is drawn from
 *   q(n) = [0.95 kappa cosh(kappa mu.n) / sinh(kappa) + 0.05] / (4 pi)
 * (antipodally symmetrised von Mises-Fisher plus 5 % uniform) and accepted with probability
 * min(1, exp(-dE/T) q(n_old) / q(n_new)); q does not depend on the site's own director, so the Boltzmann
 * distribution stays exact for any weights. Weights and hidden activations are rounded to BF16, sums are FP32. */
typedef struct mcl_mlp {
  float w1[64][7]; /* [out][in] */
  float b1[64];
  float w2[64][64];
  float b2[64];
  float w3[4][64];
  float b3[4];
} mcl_mlp;

/* Sweeps of this engine use the learned proposal with these weights (copied; NULL returns to the plain
 * proposal). While it is set, ang_var is not adapted and the acceptance in the series is that of the learned
 * moves. Every site gets one learned trial per sweep, colour by colour (no separate n -> -n trial: the proposal is
 * symmetric under n -> -n). */
int mcl_set_proposal(mcl_engine *e, const mcl_mlp *mlp, float kappa_max);
/* Mixture of the learned and the plain sweep (no counterpart in the reference): with a proposal set, one learned
 * sweep after every period - 1 plain sweeps, counted across mcl_sweeps calls from this call on; period 1 (the
 * default) makes every sweep learned. Each sweep is an exact Metropolis(-Hastings) kernel of the same distribution,
 * so the cycle leaves it exact. The plain sweeps adapt ang_var or not as mcl_set_adaptation says. */
int mcl_set_proposal_mix(mcl_engine *e, int period);
/* ang_var adaptation after each sweep (default 1, as the reference, src/evolve.cu:302-313). 0 keeps the plain
 * proposal's amplitude fixed: the fixed-amplitude yardstick of autocorrelation comparisons. */
int mcl_set_adaptation(mcl_engine *e, int enable);
/* Training samples from the current state of one replica: n sites drawn with Philox(seed, sample index). Device
 * buffers: d_features n x 8 floats (7 features, then 1 for a non-empty site / 0 for an empty one), d_directors
 * n x 3 floats (the site's director). Synchronises. */
int mcl_extract_samples(mcl_engine *e, int replica, long long n, unsigned long long seed, float *d_features,
                        float *d_directors);
/* The tensor-core MLP on n feature rows (device, n x 8 floats as above) -> d_out n x 4 raw outputs (before the
 * normalisation of mu and the softplus of kappa). Synchronises `stream`. */
int mcl_mlp_forward(const mcl_mlp *mlp, const float *d_features, long long n, float *d_out, void *stream);
/* The same on Blackwell's tcgen05 tensor cores (operands in shared memory, accumulators in tensor memory, 256 rows
 * per CTA); identical operand rounding, FP32 sums in another order. MCL_ERR_CUDA if a tensor-core completion does
 * not arrive within 2 s (the CTA frees its tensor memory and stops). */
int mcl_mlp_forward_tcgen05(const mcl_mlp *mlp, const float *d_features, long long n, float *d_out, void *stream);

/* Training on the GPU (no counterpart in the reference): loss = -mean log(4 pi q(n | features)) over samples (maximum likelihood of the site's
 * conditional distribution), Adam (beta 0.9 / 0.999, eps 1e-8) on FP32 master weights, BF16-rounded weights in
 * the passes. Batches are device buffers in the mcl_extract_samples format, at most max_batch rows. */
typedef struct mcl_trainer mcl_trainer;
int mcl_trainer_create(const mcl_mlp *init, long long max_batch, float kappa_max, mcl_trainer **out);
/* Gradient of the mean loss at the current weights (no update) and the loss. Synchronises. */
int mcl_trainer_gradient(mcl_trainer *t, const float *d_features, const float *d_directors, long long n,
                         mcl_mlp *grad, double *loss);
/* One Adam step with learning rate lr; loss (may be NULL) is the batch loss before the step. */
int mcl_trainer_step(mcl_trainer *t, const float *d_features, const float *d_directors, long long n, float lr,
                     double *loss);
int mcl_trainer_get(mcl_trainer *t, mcl_mlp *out);
int mcl_trainer_destroy(mcl_trainer *t);

/* Observables of a bulk or slab lattice whose directors already lie in device memory, computed without allocating
 * anything. No counterpart in the reference. mcl_measure needs an engine, and mcl_create allocates the engine's
 * buffers; this function serves callers that hold the directors in their own device buffer and cannot allocate
 * when they measure, such as a program whose pool allocator has reserved the device's memory, or a loop that
 * must not absorb the device-wide synchronisation of cudaMalloc/cudaFree.
 *   d_ni     3 floats per site, site (i, j, k) at index i + Nx (j + Ny k), in memory of the current device (or
 *            managed memory); its allocation must hold all 3 Nx Ny Nz floats (checked).
 *   out      host struct: energy, q, S, director, nsum and n_valid as mcl_measure gives them (within FP64
 *            rounding of the sums); acceptance 0, ang_var = replica->ang_var, sweep 0. replica->T and seed are
 *            not used.
 *   stream   cudaStream_t the two kernels run on (NULL: the default stream); the call waits for that stream.
 * Limits: at most 2^26 = 67,108,864 sites; larger lattices return MCL_ERR_ARG (the partial sums go to a fixed
 * 1.25 MiB array in the library's device memory). Sphere and custom geometries return MCL_ERR_ARG.
 * The first call on each device looks up that array's address (cudaGetSymbolAddress), which may load the
 * library's device code; make that first call before any stream capture on the device. The device must not be
 * reset (cudaDeviceReset) afterwards. Nothing in the array needs to start at zero. There is one array per device:
 * calls on the same device must not overlap (from several host threads, or on several streams); they would
 * overwrite each other's partial sums. */
int mcl_observe_device(const mcl_model *model, const mcl_replica *replica, const float *d_ni, mcl_observables *out,
                       void *stream);

/* Message of the last failed call on this thread ("" if none). */
const char *mcl_last_error(void);
/* Library version string. */
const char *mcl_version(void);

#ifdef __cplusplus
}
#endif
#endif
