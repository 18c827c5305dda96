"""Benchmark of the checkerboard Metropolis sweep on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mclics_b200|reference]

Workload: the GHRL slab of 256 x 256 x 256 sites (x, y periodic, z free), K11:K22:K33 = 1 : 0.5 : 1.5,
homeotropic anchoring W = 1.5 on both plates, T = 0.8, initial director (0, 0, 1) plus uniform noise of amplitude
0.1 per component (seed 7), FP32 directors, FP64 reductions. One step = one Monte Carlo sweep of all sites plus its
measurement (energy, Q tensor, S, acceptance, device-side ang_var adaptation), i.e. one measurement sweep of the
reference's thermalGPU loop. Metric: site updates per second (whole job, all GPUs).

  value      device time (CUDA events on the engine's stream) of K steps with the lattice resident in HBM. The
             lattice (211 MB padded) is larger than L2 (126 MB), so no flush is needed between steps. The tile
             plan is chosen by mcl_autotune before timing, and the K steps are one mcl_sweeps call replaying a
             captured CUDA graph of the sweeps.
  e2e        the same steps through the C ABI, one mcl_sweeps_io call per step as a drop-in caller makes it, host
             buffers and host<->device transfers inside the timed region: the step's input (the temperature of
             every replica) goes up from the engine's mapped pinned staging, the sweep runs, and the step's result
             (the observables record of every replica and the kernels' two error words) comes down into it; one
             host synchronisation per step.
  e2e_reference_data_movement  the same, plus the whole director field down every step, as the reference's GPU
             loop moves it (it computes Q on the host after every measurement sweep, src/evolve_thermal.cu:90;
             this engine computes it on the device, so a caller needs the field only for snapshots).
  roofline   the sweep kernel(s) only: algorithmic 24 B per site update (one FP32 director read + write) per
             sweep / kernel time, against the measured HBM copy bandwidth.
  cpu_baseline  the reference's own OpenMP CPU sweep + measurement (oracle/_ref/mclics_ref_timing, built from the
             reference sources) on all host cores, on a bounded sample of the same lattice (of the workload's
             replicas, for --workload cN).

--impl reference times that reference CPU path alone (rank 0) and prints its line with "impl": "reference"; with
--workload cN it times that workload's replicas (one after another, from the GPU arm's initial directors).
--impl reference-gpu and --impl dropin are context lines: the reference's own GPU program, and that program with
this library behind its GPU modes, timed as whole programs by the reference's differencing method.
Multi-GPU (torchrun): every rank sweeps its own independent replica of the workload (no data-path collective;
"scaling": "weak"); value = all ranks' site updates / the slowest rank's device time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_SITE_UPDATE = 24
TIMED_TARGET_MS = 300.0  # the device-timed K-step region is repeated until the repeats span about this long
MAX_REPEATS = 50
METRIC = "site-updates/s"
SEED = 7


def c3_sizes(seed=11, n=64):
    """C3's replica sizes: L = 2 round(exp(U(ln 16, ln 128)) / 2) from a seeded numpy stream."""
    rng = np.random.default_rng(seed)
    return [int(2 * round(np.exp(rng.uniform(np.log(16), np.log(128))) / 2)) for _ in range(n)]


def workload(name):
    """Model, replicas and descriptive config of a named workload (synthetic lattices of the configs' shapes)."""
    import mclics_b200 as M
    if name == "c2":
        model = M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=[("homeotropic", 1.5, 0, 0)] * 2)
        reps = [dict(nx=256, ny=256, nz=256, geometry="slab", periodic=(1, 1, 0), T=0.8, seed=7)]
        cfg = {"workload": "ghrl_slab_256^3_k1:0.5:1.5_homeotropic_W1.5_T0.8", "geometry": "slab",
               "potential": "ghrl", "lattices": "1 x 256^3", "k11_k22_k33": [1, 0.5, 1.5],
               "anchoring": "homeotropic W=1.5 (both plates)", "T": 0.8}
        ic = "z_noise"
    elif name == "c1":
        model = M.Model("ll")
        reps = [dict(nx=32, ny=32, nz=32, geometry="bulk", periodic=(1, 1, 1), T=1.1, seed=1)]
        cfg = {"workload": "ll_bulk_32^3_T1.1", "potential": "ll", "lattices": "1 x 32^3", "T": 1.1}
        ic = "random"
    elif name == "c3":
        sizes = c3_sizes()
        model = M.Model("ll")
        reps = [dict(nx=L, ny=L, nz=L, geometry="bulk", periodic=(1, 1, 1), T=1.0 + 0.2 * r / 63, seed=r + 1)
                for r, L in enumerate(sizes)]
        cfg = {"workload": "ll_64_replicas_16^3-128^3_T1.00-1.20", "potential": "ll",
               "lattices": "64 replicas, L from 2 round(exp(U(ln16, ln128))/2), seed 11",
               "sites": int(sum(L ** 3 for L in sizes))}
        ic = "random"
    elif name == "c4":
        model = M.Model("ll")
        reps = [dict(nx=128, ny=128, nz=128, geometry="bulk", periodic=(1, 1, 1), T=T, seed=3 + i)
                for i, T in enumerate((0.3, 0.8, 1.12))]
        cfg = {"workload": "ll_bulk_128^3_T0.3_0.8_1.12", "potential": "ll", "lattices": "3 x 128^3 (one per T)"}
        ic = "random"
    elif name == "c5":
        model = M.Model("pear", field_dir=(0, 0, 1), elecP=1.0, surfaces=[("fg", 1.0, 0, 0)] * 2)
        reps = [dict(nx=256, ny=256, nz=64, geometry="slab", periodic=(1, 1, 0), T=0.5, elecE=2.0 * i / 31, seed=5 + i)
                for i in range(32)]
        cfg = {"workload": "pear_slab_256x256x64_32_fields_0-2_T0.5", "potential": "pear", "geometry": "slab",
               "lattices": "32 replicas (field 0..2 along z, elecP=1, fg W=1)", "T": 0.5}
        ic = "random"
    else:
        raise SystemExit("unknown workload " + name)
    return model, reps, cfg, ic


def initial_state(n, kind, seed):
    rng = np.random.default_rng(seed)
    if kind == "z_noise":  # (0, 0, 1) + uniform noise of amplitude 0.1 per component, renormalised
        v = rng.uniform(-0.1, 0.1, size=(n, 3)).astype(np.float32)
        v[:, 2] += 1.0
    else:
        v = rng.normal(size=(n, 3)).astype(np.float32)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v.reshape(-1).astype(np.float32)


def c2_input_text():
    return ("Nx 256\nNy 256\nNz 256\ngeometry slab\nxbound periodic\nybound periodic\npotential ghrl\nk11 1\nk22 0.5\n"
            "k33 1.5\nanchoring_type 0 homeotropic\nW 0 1.5\nanchoring_type 1 homeotropic\nW 1 1.5\nevol thermal\n"
            "Ti 0.8\nTf 0.8\ndT -0.1\nMCT 200\nMCS 1000\nic homogeneous\ntheta_0 0\nphi_0 0\nseed 7\n")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload, plan):
    """Per-launch DRAM bytes of the sweep kernel from the committed ncu summary (profiles/ncu_traffic.json), when
    the summary was taken with exactly this run's plan ("tile configuration,planes per segment"); None otherwise."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        caps = json.load(f).get(workload) or []
    for d in caps if isinstance(caps, list) else [caps]:  # one capture per plan the autotuner has been seen to pick for this workload
        if d["plan"] == plan:
            return d["dram_bytes_per_launch"]
    return None


class ClockSampler:
    """SM clock and clock-event reasons of this rank's GPU, sampled every 10 ms through NVML while the timed
    regions run (nvidia-smi every 200 ms when NVML is unavailable). The GPU is found by the UUID torch reports,
    so CUDA_VISIBLE_DEVICES reordering does not matter."""

    REASONS = [("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80)]
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, set of reason names)
        self.source = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            try:
                h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
            self._nvml = (pynvml, h, pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.source = "nvml"
        except Exception:
            self._nvml = None
            self.source = "nvidia-smi"

    def _sample(self):
        if self._nvml:
            nv, h, mx = self._nvml
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            try:
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.samples.append((float(sm), float(mx), {n for n, b in self.REASONS if bits & b}))
            return 0.01
        out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=5).stdout.strip()
        if out:
            s = [x.strip() for x in out.split(",")]
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            rs = {n for k, n in enumerate(names) if len(s) > 5 + k and s[5 + k].lower().startswith("active")}
            if s[1].replace(".", "").isdigit() and s[2].replace(".", "").isdigit():
                self.samples.append((float(s[1]), float(s[2]), rs))
        return 0.2

    def start(self):
        self._stop.clear()

        def loop():
            while not self._stop.is_set():
                try:
                    dt = self._sample()
                except Exception:
                    dt = 0.2
                self._stop.wait(dt)
        self._t = threading.Thread(target=loop, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0,
                    "source": self.source}
        reasons = set()
        for s in self.samples:
            reasons |= s[2]
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": self.source,
                "region": "device-timed and end-to-end-timed steps"}


def reference_input_text(name, rep):
    """The reference's input file for one replica of a workload: the lattice, physics, temperature and field of the
    GPU arm's replica (the timing harness runs at T = Ti and, in the electric mode, at the field Ei)."""
    if name == "c2":
        return c2_input_text()
    lines = ["Nx %d" % rep["nx"], "Ny %d" % rep["ny"], "Nz %d" % rep["nz"], "geometry %s" % rep["geometry"],
             "xbound periodic", "ybound periodic", "seed %d" % rep["seed"], "ic random", "MCT 0", "MCS 1"]
    if rep["geometry"] == "bulk":
        lines.append("zbound periodic")
    if name in ("c1", "c3", "c4"):
        lines += ["potential ll", "evol thermal", "Ti %r" % rep["T"], "Tf %r" % rep["T"], "dT -0.1"]
    elif name == "c5":
        lines += ["potential pear", "A 1.0", "B1 0.04", "C 0.3", "anchoring_type 0 fg", "W 0 1.0",
                  "anchoring_type 1 fg", "W 1 1.0", "elecX 0", "elecY 0", "elecZ 1", "elecP 1.0", "evol electric",
                  "Ti %r" % rep["T"], "Ei %r" % rep["elecE"], "Ef %r" % rep["elecE"], "dE 0.1"]
    else:
        raise SystemExit("no reference input for workload " + name)
    return "\n".join(lines) + "\n"


def reference_cpu(steps, warmup, budget_s=150.0, name="c2"):
    """Times the reference's own CPU sweep + measurement (oracle/_ref/mclics_ref_timing) on all host cores, on the
    replicas of a workload, each from the GPU arm's own initial directors (passed as a raw file, bit for bit). One
    step = one measured sweep of every timed replica, the replicas one after another. The requested warm-up sweeps
    run untimed; the timed sweeps are bounded by budget_s: a probe sweep of the largest replica sizes the sample, and
    when one step of all replicas would not fit the budget with its warm-up, every m-th replica is timed."""
    exe = os.path.join(ROOT, "oracle", "_ref", "mclics_ref_timing")
    if not os.path.exists(exe):
        return None, "oracle/_ref/mclics_ref_timing not built"
    import shutil
    import tempfile
    _, reps, _, ic = workload(name)
    sizes = [r["nx"] * r["ny"] * r["nz"] for r in reps]
    cores = os.cpu_count() or 1
    d = tempfile.mkdtemp(prefix="mcl_ref_")
    try:
        env = dict(os.environ, OMP_NUM_THREADS=str(cores))

        def run(i, w, k):
            with open(os.path.join(d, "input.txt"), "w") as f:
                f.write(reference_input_text(name, reps[i]))
            initial_state(sizes[i], ic, SEED + 97 * i).tofile(os.path.join(d, "start.f32"))
            p = subprocess.run([exe, "input.txt", str(w), str(k), "1", "0", str(SEED), "start.f32"], cwd=d, env=env,
                               capture_output=True, text=True, timeout=900)
            if p.returncode != 0:
                raise RuntimeError(p.stderr[-500:])
            return json.loads(p.stdout.strip().splitlines()[-1])

        big = max(range(len(reps)), key=lambda i: sizes[i])
        per_site = max(run(big, 0, 1)["seconds"], 1e-4) / sizes[big]
        m = max(1, math.ceil(per_site * sum(sizes) * (warmup + 1) / budget_s))
        chosen = list(range(0, len(reps), m))
        per_step = per_site * sum(sizes[i] for i in chosen)
        k = max(1, min(steps, int(budget_s / per_step) - warmup))
        runs = [run(i, warmup, k) for i in chosen]
    finally:
        shutil.rmtree(d, ignore_errors=True)
    r = {"steps": k, "seconds": sum(x["seconds"] for x in runs), "threads": runs[0]["threads"],
         "sites": sum(sizes[i] for i in chosen), "replicas_timed": len(chosen), "replicas": len(reps),
         "replica_stride": m, "steps_requested": steps, "warmup": warmup}
    return r, None


def reference_sample(r, name):
    """The sample a reference_cpu result covers, in words."""
    which = ("the 256^3 lattice" if name == "c2" else
             "all %d replicas" % r["replicas"] if r["replicas_timed"] == r["replicas"] and r["replicas"] > 1 else
             "the lattice" if r["replicas"] == 1 else
             "%d of the %d replicas (every %d-th)" % (r["replicas_timed"], r["replicas"], r["replica_stride"]))
    return ("%d measured sweep%s of %s after %d warm-up sweep%s, from the GPU arm's initial directors (reference "
            "EvolveN::Monte_Carlo_Step + energy_calculator + Q_tensor + eigen, GSL replaced by the shim)"
            % (r["steps"], "" if r["steps"] == 1 else "s", which, r["warmup"], "" if r["warmup"] == 1 else "s"))


def c2_program_text(mct, mcs):
    """C2's input for the reference's program in its GPU thermal mode, with mct thermalisation and mcs measured
    sweeps."""
    text = c2_input_text().replace("evol thermal", "evol thermalGPU")
    return text.replace("MCT 200", "MCT %d" % mct).replace("MCS 1000", "MCS %d" % mcs)


def program_runs(exe, k_meas, k_therm, k0=200, repeats=2, text_for=c2_program_text, sites=256 ** 3):
    """The reference's differencing method on a whole program (paper/benchmark: the fastest of the repetitions of a
    run with more sweeps minus the fastest of a run with fewer): GPU-mode runs of one input (text_for(MCT, MCS);
    the 256^3 GHRL slab by default), all with at least k0 thermalisation sweeps, with 1 + k_meas and with 1 measured sweep, and with k0 + k_therm
    thermalisation sweeps. The k0 sweeps give every run the same kind of final field: the snapshot writer
    (src/io.cpp:59-89, a %g line and a local order parameter per site) takes seconds longer on a thermalised field
    than on the homogeneous start, which a base run of one sweep would still be close to. Every run writes ic.csv
    and one snapshot (about 1 GB each for 256^3), so the runs go to /dev/shm where it exists: on disk their write
    time varies by seconds between runs, more than the sweeps being measured."""
    import shutil
    import tempfile
    where = None
    if os.path.isdir("/dev/shm") and shutil.disk_usage("/dev/shm").free > 8 * 2 ** 30:  # two 1 GB files per run
        where = "/dev/shm"

    def run(mct, mcs):
        best = None
        for _ in range(repeats):
            d = tempfile.mkdtemp(prefix="mcl_prog_", dir=where)
            try:
                with open(os.path.join(d, "input.txt"), "w") as f:
                    f.write(text_for(mct, mcs))
                t0 = time.perf_counter()
                p = subprocess.run([exe, "input.txt"], cwd=d, capture_output=True, text=True, timeout=1200,
                                   env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)))
                t = time.perf_counter() - t0
                if p.returncode != 0:
                    raise RuntimeError(p.stderr[-500:])
            finally:
                shutil.rmtree(d, ignore_errors=True)
            best = t if best is None else min(best, t)
        return best

    base = run(k0, 1)
    meas = run(k0, 1 + k_meas)
    therm = run(k0 + k_therm, 1)
    return {"measured_s_per_sweep": (meas - base) / k_meas, "thermalisation_s_per_sweep": (therm - base) / k_therm,
            "sites": sites, "steps": k_meas, "thermalisation_sweeps": k_therm, "base_thermalisation_sweeps": k0,
            "runs_s": [base, meas, therm], "repeats": repeats, "run_dir": where or "default temporary directory"}


def program_method(r):
    """The keys that describe a program_runs measurement in a context line."""
    return {"method": "wall time of thermalGPU runs with K0 thermalisation sweeps and 1 + K or 1 measured sweeps, and "
                      "with K0 + K2 thermalisation sweeps and 1 measured sweep, the fastest of %d each, differenced; "
                      "run directory %s" % (r["repeats"], r["run_dir"]),
            "base_thermalisation_sweeps": r["base_thermalisation_sweeps"],
            "thermalisation_sweeps": r["thermalisation_sweeps"], "runs_s": r["runs_s"]}


def dropin(steps):
    """Context: the compiled drop-in (the reference's own program with this library behind its *EvolveNGPU classes,
    mclics_b200/adapter/_build/mclics_dropin) on the same input and by the same method as reference_gpu."""
    exe = os.path.join(ROOT, "mclics_b200", "adapter", "_build", "mclics_dropin")
    if not os.path.exists(exe):
        return None, "mclics_b200/adapter/_build/mclics_dropin not built (make -C mclics_b200/adapter REF=...)"
    return program_runs(exe, max(steps, 20000), max(steps, 20000)), None


# Sweeps per difference of the reference GPU program, by workload: (measured, thermalisation). Each difference
# must stand well above the run-to-run noise of one program run (its set-up and its ic.csv and snapshot files).
REFERENCE_GPU_SWEEPS = {"c1": (2000, 20000), "c2": (20, 1000), "c4": (40, 4000)}


def reference_gpu(steps, variant, name="c2"):
    """Context, not the reference arm: the reference's own GPU program (its .cu path, oracle/_ref/mclics_ref_gpu
    built for sm_100, or mclics_ref_gpu_jit as shipped, PTX compiled by the driver), timed by the reference's own
    differencing (paper/benchmark: a run with more sweeps minus a run with fewer). Measured sweeps (the GPU thermal
    mode's MCS loop: sweep, energy, lattice copied to the host, Q tensor and S there) and thermalisation sweeps (MCT:
    the eight sublattice launches and the acceptance reduction only) separately. One program is one lattice, so a
    workload of several replicas is one program per replica, their per-sweep times added. On C2 the reference has
    no noisy initial condition, so it starts from (0, 0, 1); the others start from its own random directors. C3 and
    C5 (64 and 32 programs, three runs each, twice) are not timed."""
    exe = os.path.join(ROOT, "oracle", "_ref", "mclics_ref_gpu" if variant == "sm_100" else "mclics_ref_gpu_jit")
    if not os.path.exists(exe):
        return None, "%s not built (make -C oracle REF=... refgpu)" % os.path.relpath(exe, ROOT)
    if name not in REFERENCE_GPU_SWEEPS:
        return None, "not timed for workload %s: one reference program per replica (%s)" % (
            name, "64 programs" if name == "c3" else "32 programs")
    if name == "c2":
        return program_runs(exe, steps, max(steps, 1000)), None
    k_meas, k_therm = REFERENCE_GPU_SWEEPS[name]
    _, reps, _, _ = workload(name)
    parts = []
    for rep in reps:
        base_text = reference_input_text(name, rep).replace("evol thermal", "evol thermalGPU")

        def text_for(mct, mcs, base_text=base_text):
            return base_text.replace("MCT 0", "MCT %d" % mct).replace("MCS 1", "MCS %d" % mcs)

        parts.append(program_runs(exe, max(steps, k_meas), k_therm, k0=200, text_for=text_for,
                                  sites=rep["nx"] * rep["ny"] * rep["nz"]))
    r = dict(parts[0])
    r["sites"] = sum(x["sites"] for x in parts)
    r["measured_s_per_sweep"] = sum(x["measured_s_per_sweep"] for x in parts)
    r["thermalisation_s_per_sweep"] = sum(x["thermalisation_s_per_sweep"] for x in parts)
    r["runs_s"] = [x["runs_s"] for x in parts] if len(parts) > 1 else parts[0]["runs_s"]
    return r, None


def gpu_arm(args, rank, world, local_rank):
    import torch
    import mclics_b200 as M

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    model, reps, cfg, ic = workload(args.workload)
    all_sites = sum(r["nx"] * r["ny"] * r["nz"] for r in reps)
    if args.shard and world > 1:  # strong scaling: this rank's share of the batch, largest replicas first
        from mclics_b200 import sharding
        if len(reps) < world:
            raise SystemExit("--shard needs at least one replica per rank (%d replicas, %d ranks)" % (len(reps), world))
        reps = [reps[i] for i in sharding.shard([r["nx"] * r["ny"] * r["nz"] for r in reps], world, rank)]
        creps = [M.Replica(**r) for r in reps]
    else:  # weak scaling: every rank sweeps its own copy of the workload
        creps = [M.Replica(**dict(r, seed=r["seed"] + 1000 * rank)) for r in reps]
    eng = M.Engine(model, creps)
    sizes = [r["nx"] * r["ny"] * r["nz"] for r in reps]
    for i, n in enumerate(sizes):
        eng.upload(i, initial_state(n, ic, SEED + 97 * i + rank))
    stream = torch.cuda.Stream(device=dev)
    eng.set_stream(stream.cuda_stream)
    sites = sum(sizes)

    for _ in range(args.warmup):
        eng.sweeps(1, measure=True)
    eng.synchronize()
    # tile plan by the autotuner (state restored) or given by --plan, then graph replay of the sweeps
    if args.plan:
        cfg_s, _, seg_s = args.plan.partition(",")
        eng.set_plan(int(cfg_s), int(seg_s or 0))
        tuning = dict(eng.plan(), candidates=0)
    else:
        tuning = eng.autotune(10)  # 10 sweeps per candidate: plans within 1 % of each other need them
    # every record the timed regions append (device steps, profiled sweeps, two end-to-end loops with warm-up)
    # fits the series, so no timed sweep reallocates it or captures its graph again
    eng.reserve_series(eng.series_length() + (2 * MAX_REPEATS + 4) * args.steps + 256)
    eng.set_graphs(True)
    eng.sweeps(2, measure=True)  # captures the graph outside the timed region
    eng.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed_steps():
        """One timed region: exactly K steps (K sweeps, each with its measurement), events on the engine's stream,
        a barrier over the ranks and a device synchronisation on both sides."""
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0.record(stream)
        eng.sweeps(args.steps, measure=True)
        e1.record(stream)
        e1.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # A short K (the driver runs K = 20: ~5 ms) gives a timed region of a few ms, so the region is repeated until
    # the repeats span about TIMED_TARGET_MS (at most MAX_REPEATS), and the median is reported.
    _, _, l0 = eng.profile_read()
    dev_all = [timed_steps()]
    _, _, l1 = eng.profile_read()
    launches = l1 - l0
    repeats = torch.tensor([float(min(MAX_REPEATS, max(1, math.ceil(TIMED_TARGET_MS / max(dev_all[0], 1e-3)))))],
                           dtype=torch.float64, device=dev)
    if world > 1:  # every rank runs the same number of repeats
        torch.distributed.all_reduce(repeats, op=torch.distributed.ReduceOp.MAX)
    for _ in range(int(repeats.item()) - 1):
        dev_all.append(timed_steps())
    clocks.stop()
    dev_ms = statistics.median(dev_all)
    # sweep-kernel time for the roofline: a separate run with per-sweep events (direct launches)
    eng.profile(True)
    ms0, n0, _ = eng.profile_read()
    eng.sweeps(min(args.steps, 50), measure=True)
    eng.synchronize()
    ms1, n1, _ = eng.profile_read()
    eng.profile(False)
    kernel_ms = (ms1 - ms0) / max(1, n1 - n0)
    rec = eng.series(0, eng.series_length() - 1, 1)[0]

    # end to end through the C ABI with host buffers, all replicas: temperatures up, the step's observables down
    # (and, second, also the whole director field down every step, the reference GPU loop's data movement)
    host_ni = [torch.empty(3 * n, dtype=torch.float32, pin_memory=True) for n in sizes]
    host_T = np.array([r["T"] for r in reps], dtype=np.float32)
    host_obs = np.zeros(len(reps), M.OBS_DTYPE)

    def e2e_loop(lattice_down, n_repeats):
        for _ in range(max(3, min(args.warmup, 10))):  # untimed: staging allocation, first launches
            eng.sweeps_io(1, host_T, host_obs)
            if lattice_down:
                for i in range(len(reps)):
                    M.check(M.lib().mcl_download_directors(eng._h, i, host_ni[i].data_ptr()))
        times = []
        for _ in range(n_repeats):  # each repeat times exactly K steps; the median is reported
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                eng.sweeps_io(1, host_T, host_obs)  # temperatures up, one measured sweep, its records down
                if lattice_down:
                    for i in range(len(reps)):
                        M.check(M.lib().mcl_download_directors(eng._h, i, host_ni[i].data_ptr()))
            times.append(time.perf_counter() - t0)
        return statistics.median(times)

    clocks.start()
    e2e_s = e2e_loop(False, int(repeats.item()))
    e2e_lat_s = e2e_loop(True, 1)
    clocks.stop()

    times = torch.tensor([dev_ms, e2e_s * 1e3, e2e_lat_s * 1e3], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(times, op=torch.distributed.ReduceOp.MAX)
    dev_ms_max, e2e_ms_max, e2e_lat_ms_max = float(times[0]), float(times[1]), float(times[2])
    eng.close()
    return dict(dev_ms=dev_ms_max, e2e_ms=e2e_ms_max, e2e_lat_ms=e2e_lat_ms_max, kernel_ms=kernel_ms,
                timed_repeats=int(repeats.item()), dev_ms_all=dev_all,
                launches=launches, sites=sites,
                all_sites=all_sites,
                n_rep=len(reps), clocks=clocks.summary(), S=float(rec["S"]), E=float(rec["energy"]),
                acc=float(rec["acceptance"]), cfg=cfg, tuning=tuning)


def zslab_arm(args, rank, world, local_rank):
    """The workload's first lattice split along z over the ranks (mclics_b200.zslab): every rank sweeps its planes
    with the colour passes and exchanges its boundary planes after each pass (NCCL send/recv through
    torch.distributed), one FP64 all-reduce of the sums per sweep. Strong scaling: the lattice is the same for
    every N. Device time of K measured sweeps, max over ranks."""
    import torch
    from mclics_b200 import zslab
    torch.cuda.set_device(local_rank)
    model, reps, cfg, ic = workload(args.workload)
    r0 = reps[0]
    nx, ny, nz = r0["nx"], r0["ny"], r0["nz"]
    per, geo = r0.get("periodic", (1, 1, 1)), r0.get("geometry", "bulk")
    slab = zslab.ZSlab(model, nx, ny, nz, rank, world, zslab.TorchExchange(), geometry=geo, periodic_xy=per[:2],
                       periodic_z=bool(per[2]) and geo != "slab", T=r0["T"], seed=r0["seed"])
    slab.upload_global(initial_state(nx * ny * nz, ic, SEED))  # the same global lattice on every rank
    slab.sweeps(args.warmup, measure=True)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(slab.stream)
    slab.sweeps(args.steps, measure=True)
    e1.record(slab.stream)
    e1.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.stop()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    rec = slab.series()[-1]
    out = dict(dev_ms=float(t[0]), sites=nx * ny * nz, nz_own=slab.nz_own, cfg=cfg, clocks=clocks.summary(),
               plan=slab.eng.plan(), S=float(rec["S"]), E=float(rec["energy"]), acc=float(rec["acceptance"]))
    slab.eng.close()
    return out


def zslab_main(args, rank, world, local_rank):
    import torch
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res = zslab_arm(args, rank, world, local_rank)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_kind = measured_peaks()
    sec = res["dev_ms"] / 1e3
    achieved = res["sites"] * BYTES_PER_SITE_UPDATE * args.steps / sec / world / 1e9  # per GPU
    config = dict(res["cfg"], step="1 sweep + measurement of the whole lattice",
                  parallelism="one lattice split along z over %d GPUs (%d planes on rank 0)" % (world, res["nz_own"]),
                  decomposition="z-slab: boundary planes exchanged after each colour pass, 11-double all-reduce "
                                "per sweep", plan=res["plan"], global_sites_per_step=res["sites"])
    line = {
        "metric": METRIC, "value": res["sites"] * args.steps / sec, "unit": "site-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["dev_ms"] / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config, "mode": "zslab",
        "e2e": None, "e2e_note": "device-timed only: the z-slab mode measures the decomposition, not host transfers",
        "gpu_launches": 8 * args.steps,  # per sweep: 2 passes, 2 packs, 2 unpacks, sums, finalisation
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": None, "per": "GPU"},
        "clocks": res["clocks"],
        "physics": {"S_last": res["S"], "E_last": res["E"], "acceptance_last": res["acc"]},
    }
    print(json.dumps(line))
    return 0


def learned_compare(args):
    """Learned vs plain proposal on one workload (c4: LL 128^3 at T = 0.3, 0.8, 1.12): the network is trained on
    the GPU from plain-sweep states (seed 3), then both proposals run the same number of measured sweeps from the
    same equilibrated start, and the integrated autocorrelation times of E and S (Sokal windowing) give effective
    samples per device second. The plain arm keeps ang_var fixed at its adapted value (the fixed-amplitude
    proposal the learned one is measured against)."""
    import torch
    import mclics_b200 as M
    from mclics_b200 import analysis, learned

    model, reps, cfg, _ = workload(args.workload)
    creps = [M.Replica(**r) for r in reps]
    sizes = [r["nx"] * r["ny"] * r["nz"] for r in reps]
    Ts = [r["T"] for r in reps]
    # one label per replica: its temperature, and its field where the replicas differ in field (c5)
    fields = [r.get("elecE", 1.0) for r in reps]
    labels = ["T=%g" % T if len(set(fields)) == 1 else "T=%g,E=%.4g" % (T, E) for T, E in zip(Ts, fields)]

    def engine(seed_off):
        e = M.Engine(model, creps, M.SCHED_CHECKER2)
        for i, n in enumerate(sizes):  # ordered start: the nematic states equilibrate within the thermalisation
            e.upload(i, initial_state(n, "z_noise", 1000 + i + seed_off))
        return e

    t0 = time.perf_counter()
    tr = engine(0)
    tr.sweeps(500)
    snaps = 20
    per = max(1, args.train_samples // (snaps * len(reps)))
    feat, dirs = learned.collect(tr, snapshots=snaps, gap=10, per_snapshot=per, seed=3)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    params, losses = learned.train(feat, dirs, epochs=3, batch=8192, seed=3)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    tr.close()
    n_samples = int(feat.shape[0])
    del feat, dirs

    stream = torch.cuda.Stream()
    K = args.ess_sweeps
    arms = {}
    mixes = [int(k) for k in args.mix.split(",") if k.strip() and int(k) > 1]
    for arm in ["plain", "learned"] + ["mix%d" % k for k in mixes]:
        e = engine(7)
        e.set_stream(stream.cuda_stream)
        e.sweeps(args.therm_sweeps)  # ~10 tau_E at T = 1.12 (tau_E ~ 500 sweeps for the plain proposal)
        e.set_adaptation(False)  # every plain sweep at the amplitude adapted during the thermalisation
        if arm != "plain":
            e.set_proposal(params)
            if arm.startswith("mix"):  # one learned sweep after every k - 1 plain ones
                e.set_proposal_mix(int(arm[3:]))
            e.sweeps(100)
        e.clear_series()
        e.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e.sweeps(K, measure=True)
        ev1.record(stream)
        ev1.synchronize()
        sec = ev0.elapsed_time(ev1) / 1e3
        res = {"device_s": sec, "ms_per_sweep": 1e3 * sec / K, "site_updates_per_s": sum(sizes) * K / sec}
        for i, key in enumerate(labels):
            sr = e.series(i)
            tE, wE = analysis.tau_int(sr["energy"])
            tS, wS = analysis.tau_int(sr["S"])
            mE, dE = analysis.mean_and_error(sr["energy"])
            mS, dS = analysis.mean_and_error(sr["S"])
            res[key] = {"tau_E": tE, "window_E": wE, "tau_S": tS, "window_S": wS,
                           "ess_per_s_E": K / (2 * tE) / sec, "ess_per_s_S": K / (2 * tS) / sec,
                           "E": mE, "E_err": dE, "S": mS, "S_err": dS,
                           "E_err_blocks": analysis.block_error(sr["energy"]),
                           "S_err_blocks": analysis.block_error(sr["S"]),
                           "acceptance": float(sr["acceptance"].mean())}
        arms[arm] = res
        e.close()
    def ratios(arm):
        out = {}
        for T in labels:
            p, l = arms["plain"][T], arms[arm][T]
            out[T] = {"ess_ratio_E": l["ess_per_s_E"] / p["ess_per_s_E"],
                      "ess_ratio_S": l["ess_per_s_S"] / p["ess_per_s_S"],
                      "z_E": (l["E"] - p["E"]) / float(np.hypot(l["E_err"], p["E_err"])),
                      "z_S": (l["S"] - p["S"]) / float(np.hypot(l["S_err"], p["S_err"])),
                      # the same differences over batch-means errors (16 blocks per arm: no tau estimate)
                      "z_E_blocks": (l["E"] - p["E"]) / float(np.hypot(l["E_err_blocks"], p["E_err_blocks"])),
                      "z_S_blocks": (l["S"] - p["S"]) / float(np.hypot(l["S_err_blocks"], p["S_err_blocks"]))}
        return out

    per_T = ratios("learned")
    tnis = labels[-1]  # c4: the highest temperature, T = 1.12 near T_NI
    per_arm = {arm: ratios(arm) for arm in arms if arm != "plain"}
    best = max(per_arm, key=lambda a: min(per_arm[a][tnis]["ess_ratio_E"], per_arm[a][tnis]["ess_ratio_S"]))
    line = {"metric": "ESS/s (tau_int of E and S), learned vs plain proposal, min over E and S at %s" % tnis,
            "value": min(per_T[tnis]["ess_ratio_E"], per_T[tnis]["ess_ratio_S"]), "unit": "ratio",
            "higher_is_better": True, "n_gpus": 1, "steps": K, "data": "synthetic", "dtype": "f32 / bf16 MLP",
            "config": dict(cfg, start="(0,0,1) + 0.1 uniform noise, %d thermalisation sweeps" % args.therm_sweeps,
                           sweeps_per_arm=K, tau_window="Sokal, c = 5"),
            "training": {"samples": n_samples, "collect_s": t1 - t0, "train_s": t2 - t1, "steps": len(losses),
                         "loss_first": float(losses[:20].mean()), "loss_last": float(losses[-50:].mean()),
                         "seed": 3},
            "per_T": per_T, "per_arm": per_arm, "best_arm_at_T_NI": best,
            "best_value": min(per_arm[best][tnis]["ess_ratio_E"], per_arm[best][tnis]["ess_ratio_S"]),
            "arms": arms}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="mclics_b200", choices=["mclics_b200", "reference", "reference-gpu", "dropin"])
    ap.add_argument("--reference-gpu-build", default="sm_100", choices=["sm_100", "as_shipped"],
                    help="--impl reference-gpu: the build compiled for sm_100, or the one without -arch (PTX JIT)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: split the workload's replicas across ranks (strong scaling) instead of one copy per rank")
    ap.add_argument("--learned", action="store_true",
                    help="learned vs plain proposal: train the proposal network, compare ESS/s of E and S")
    ap.add_argument("--ess-sweeps", type=int, default=120000,
                    help="--learned: measured sweeps per arm (tau_S of the plain chain is 1500-2700 sweeps on c4, "
                         "so shorter runs underestimate it)")
    ap.add_argument("--plan", default="",
                    help="tile configuration[,planes per z segment] instead of the autotuner (profiling runs)")
    ap.add_argument("--mix", default="",
                    help="--learned: also mixtures with one learned sweep every k sweeps, e.g. 2,4,8")
    ap.add_argument("--therm-sweeps", type=int, default=5000,
                    help="--learned: plain sweeps from the ordered start before both arms are measured")
    ap.add_argument("--train-samples", type=int, default=10_000_000)
    ap.add_argument("--zslab", action="store_true",
                    help="one lattice of the workload split along z over the N ranks (strong scaling)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2 (default): the headline GHRL 256^3 slab; others: the remaining configurations")
    args = ap.parse_args()
    if args.warmup < 3:  # device timing needs at least 3 untimed warm-up steps
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.learned:
        if rank != 0:
            return 0
        return learned_compare(args)
    if args.zslab and args.impl != "reference":
        return zslab_main(args, rank, world, local_rank)
    # the reference arms run the chosen workload; the drop-in's whole-program timing runs C2's input only
    _, _, config, _ = workload(args.workload if args.impl in ("mclics_b200", "reference", "reference-gpu") else "c2")
    config = dict(config, step="1 sweep + measurement of every lattice", accumulators="f64 (energy, Q, sum n)",
                  parallelism=("replicas split across %d GPUs" % args.gpus if args.shard and args.gpus > 1
                               else "independent replicas x%d" % max(1, args.gpus)))

    if args.impl == "dropin":  # context only: the reference's program with this library behind its GPU modes
        if rank != 0:
            return 0
        r, why = dropin(args.steps)
        if r is None:
            print(json.dumps({"impl": "dropin", "unavailable": why}))
            return 0
        print(json.dumps({"impl": "dropin", "metric": METRIC, "value": r["sites"] / r["measured_s_per_sweep"],
                          "unit": "site-updates/s", "n_gpus": 1, "steps": r["steps"],
                          "ms_per_step": 1e3 * r["measured_s_per_sweep"], "higher_is_better": True,
                          "config": dict(config, start="(0, 0, 1), as the reference program starts"),
                          "thermalisation_sweeps_per_s_site_updates": r["sites"] / r["thermalisation_s_per_sweep"],
                          **program_method(r)}))
        return 0

    if args.impl == "reference-gpu":  # context only: the driver's reference arm is the CPU path above
        if rank != 0:
            return 0
        r, why = reference_gpu(args.steps, args.reference_gpu_build, args.workload)
        if r is None:
            print(json.dumps({"impl": "reference-gpu", "unavailable": why}))
            return 0
        v = r["sites"] / r["measured_s_per_sweep"]
        print(json.dumps({"impl": "reference-gpu", "build": args.reference_gpu_build, "metric": METRIC, "value": v,
                          "unit": "site-updates/s", "n_gpus": 1, "steps": r["steps"],
                          "ms_per_step": 1e3 * r["measured_s_per_sweep"], "higher_is_better": True,
                          "config": dict(config, start="(0, 0, 1): the reference has no noisy initial condition"
                                         if args.workload == "c2" else "the reference program's own random directors"),
                          "thermalisation_sweeps_per_s_site_updates": r["sites"] / r["thermalisation_s_per_sweep"],
                          **program_method(r)}))
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        r, why = reference_cpu(args.steps, args.warmup, name=args.workload)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        v = r["sites"] * r["steps"] / r["seconds"]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "site-updates/s", "n_gpus": args.gpus,
                "steps": r["steps"], "warmup": r["warmup"], "steps_requested": r["steps_requested"],
                "ms_per_step": 1e3 * r["seconds"] / r["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": "site-updates/s", "cores": r["threads"], "kind": "reference",
                                 "sample": reference_sample(r, args.workload)},
                "e2e": {"value": v, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res = gpu_arm(args, rank, world, local_rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r, why = reference_cpu(10, 1, budget_s=25.0, name=args.workload)
        if r is not None:
            cpu = {"value": r["sites"] * r["steps"] / r["seconds"], "unit": "site-updates/s", "cores": r["threads"],
                   "kind": "reference", "sample": reference_sample(r, args.workload)}
        else:
            cpu = {"value": None, "unavailable": why}
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    sharded = args.shard and world > 1
    sites_total = res["all_sites"] if sharded else res["sites"] * world
    config["global_sites_per_step"] = sites_total
    tu = res["tuning"]
    config["plan"] = {"autotuned": not args.plan, "tile_config": tu["tile_config"],
                      "kernel": ("two in-place colour passes per sweep" if tu["tile_config"] >= 2 else
                                 "fused two-colour sweep (ping-pong buffers)"),
                      "rows_per_tile": tu["rows_per_tile"], "threads_per_cta": tu["threads_per_cta"],
                      "planes_per_segment": tu["planes_per_segment"], "ctas": tu["work_items"],
                      "candidates": tu["candidates"], "cuda_graph": True}
    config["l2"] = ("inputs larger than L2 (%.0f MB of directors > 126 MB)" % (res["sites"] * 12 / 1e6)
                    if res["sites"] * 12 > 126e6 else
                    "inputs smaller than L2 (%.0f MB): DRAM roofline is an upper bound" % (res["sites"] * 12 / 1e6))
    value = sites_total * args.steps / (res["dev_ms"] / 1e3)
    e2e = sites_total * args.steps / (res["e2e_ms"] / 1e3)
    e2e_lat = sites_total * args.steps / (res["e2e_lat_ms"] / 1e3)
    peak, peak_kind = measured_peaks()
    # per launch: a sweep is 2 colour-pass launches (each half the site updates) or 1 fused launch; the ratio of
    # algorithmic bytes to time is the same either way
    launches_per_sweep = 2 if tu["tile_config"] >= 2 else 1
    achieved = res["sites"] * BYTES_PER_SITE_UPDATE / (res["kernel_ms"] / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["dev_ms"] / args.steps, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
        "e2e": {"value": e2e, "unit": "site-updates/s", "h2d_bytes_per_step": 4 * res["n_rep"],
                "d2h_bytes_per_step": 144 * res["n_rep"] + 8},
        "e2e_reference_data_movement": {"value": e2e_lat, "unit": "site-updates/s",
                                        "h2d_bytes_per_step": 4 * res["n_rep"],
                                        "d2h_bytes_per_step": 144 * res["n_rep"] + 8 + 12 * res["sites"],
                                        "note": "plus the whole director field down every step, as the "
                                                "reference's GPU loop copies it for its host-side Q tensor"},
        "gpu_launches": res["launches"],
        "timing": {"repeats": res["timed_repeats"], "statistic": "median over repeats of the K-step region "
                   "(device events; end to end: host clock)", "ms_per_step_each": [t / args.steps for t in
                                                                                  res["dev_ms_all"]]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     "traffic": ncu_traffic(args.workload, "%d,%d" % (tu["tile_config"], tu["planes_per_segment"])),
                     "traffic_kind": "ncu dram read + write bytes per launch, cold L2 (profiles/ncu_traffic.json)",
                     "launches_per_sweep": launches_per_sweep,
                     "kernel_ms_per_launch": res["kernel_ms"] / launches_per_sweep,
                     "algorithmic_bytes_per_launch": res["sites"] * BYTES_PER_SITE_UPDATE / launches_per_sweep,
                     "kernel_ms_per_sweep": res["kernel_ms"],
                     "algorithmic_bytes_per_sweep": res["sites"] * BYTES_PER_SITE_UPDATE},
        "cpu_baseline": cpu,
        "clocks": res["clocks"],
        "physics": {"S_last_replica0": res["S"], "E_last_replica0": res["E"], "acceptance_last_replica0": res["acc"]},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
