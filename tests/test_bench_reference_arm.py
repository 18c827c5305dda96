"""bench.py --impl reference on the host cores: the reference's own CPU sweep + measurement (oracle/_ref) prints one
JSON line with the keys the benchmark contract asks of the reference arm, on the same metric and workload as the
GPU arm. Runs on CPU (one measured sweep of the 256^3 lattice); when oracle/_ref has not been built the arm must say
so in an "unavailable" line and exit 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        assert not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "mclics_ref_timing"))
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["metric"] == "site-updates/s" and line["unit"] == "site-updates/s" and line["higher_is_better"]
    assert line["config"]["workload"] == "ghrl_slab_256^3_k1:0.5:1.5_homeotropic_W1.5_T0.8"
    # the contract's minimum of 3 warm-up sweeps applies to this arm too, and they all run
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 3
    assert "initial directors" in line["cpu_baseline"]["sample"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_the_other_workloads():
    """--workload c1: the same contract line on C1's lattice and config (the reference arm times every workload)."""
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "c1", "--steps", "5",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    if "unavailable" in line:
        assert not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "mclics_ref_timing"))
        return
    assert line["config"]["workload"] == "ll_bulk_32^3_T1.1"
    assert line["value"] > 0 and line["steps"] == 5 and line["warmup"] == 3
    assert "5 measured sweeps of the lattice after 3 warm-up sweeps" in line["cpu_baseline"]["sample"]


def test_reference_inputs_restate_each_workload():
    """The reference input files of the batched workloads carry each replica's lattice, temperature and field."""
    sys.path.insert(0, ROOT)
    import bench
    _, reps, _, _ = bench.workload("c5")
    text = bench.reference_input_text("c5", reps[31])
    kv = dict(line.split(None, 1) for line in text.splitlines())
    assert (kv["Nx"], kv["Ny"], kv["Nz"], kv["geometry"]) == ("256", "256", "64", "slab")
    assert kv["potential"] == "pear" and kv["evol"] == "electric" and float(kv["Ei"]) == 2.0
    assert float(kv["Ti"]) == 0.5 and kv["elecP"] == "1.0" and kv["elecZ"] == "1"
    assert "anchoring_type 0 fg" in text and "anchoring_type 1 fg" in text
    _, reps, _, _ = bench.workload("c3")
    kv = dict(line.split(None, 1) for line in bench.reference_input_text("c3", reps[63]).splitlines())
    assert float(kv["Ti"]) == float(kv["Tf"]) == reps[63]["T"] and kv["zbound"] == "periodic"
    assert int(kv["Nx"]) == reps[63]["nx"]
