"""bench.py's whole-program timing (program_runs: the reference's differencing method, used for --impl reference-gpu
and --impl dropin). A stand-in program records the MCT and MCS of every run and sleeps in proportion to them; the
test checks that every run of a difference starts from the same k0 thermalisation sweeps (the snapshot at the end of
each run then has the same kind of field), that the differences recover the per-sweep costs, and that a failing
program is reported. Runs on CPU."""
import os
import stat
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

FAKE = """#!{python}
import os, sys, time
kv = dict(line.split()[:2] for line in open(sys.argv[1]) if len(line.split()) >= 2)
mct, mcs = int(kv["MCT"]), int(kv["MCS"])
with open(os.environ["FAKE_PROGRAM_LOG"], "a") as f:
    f.write("%s %d %d %s %s\\n" % (kv["evol"], mct, mcs, kv.get("Ti", "-"), kv["Nx"]))
if os.environ.get("FAKE_PROGRAM_FAIL"):
    sys.stderr.write("simulated failure\\n")
    sys.exit(3)
time.sleep(0.002 * mct + 0.004 * mcs)
"""


@pytest.fixture
def fake_program(tmp_path, monkeypatch):
    exe = tmp_path / "fake_program"
    exe.write_text(FAKE.format(python=sys.executable))
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    log = tmp_path / "runs.log"
    monkeypatch.setenv("FAKE_PROGRAM_LOG", str(log))
    return str(exe), log


def test_every_run_starts_from_the_same_thermalisation(fake_program):
    exe, log = fake_program
    r = bench.program_runs(exe, k_meas=100, k_therm=200, k0=30, repeats=2)
    runs = [line.split() for line in log.read_text().splitlines()]
    assert [x[0] for x in runs] == ["thermalGPU"] * 6
    assert [(int(x[1]), int(x[2])) for x in runs] == [(30, 1)] * 2 + [(30, 101)] * 2 + [(230, 1)] * 2
    assert r["base_thermalisation_sweeps"] == 30 and r["thermalisation_sweeps"] == 200 and r["steps"] == 100
    assert r["sites"] == 256 ** 3 and r["repeats"] == 2 and len(r["runs_s"]) == 3
    # the stand-in costs 4 ms per measured and 2 ms per thermalisation sweep; process start-up cancels in the
    # differences (fastest of two each), scheduling noise of a few ms does not matter against 0.4 s of sleep
    assert r["measured_s_per_sweep"] == pytest.approx(0.004, rel=0.25)
    assert r["thermalisation_s_per_sweep"] == pytest.approx(0.002, rel=0.25)
    keys = bench.program_method(r)
    assert keys["base_thermalisation_sweeps"] == 30 and "K0" in keys["method"]


def test_a_failing_program_is_reported(fake_program, monkeypatch):
    exe, _ = fake_program
    monkeypatch.setenv("FAKE_PROGRAM_FAIL", "1")
    with pytest.raises(RuntimeError, match="simulated failure"):
        bench.program_runs(exe, k_meas=1, k_therm=1, k0=1, repeats=1)


def test_reference_gpu_program_runs_one_program_per_replica(fake_program, tmp_path, monkeypatch):
    """--impl reference-gpu on C4: three programs (one per temperature), each differenced as above; C3 and C5 are
    reported as not timed."""
    exe, log = fake_program
    root = tmp_path / "root"
    (root / "oracle" / "_ref").mkdir(parents=True)
    os.symlink(exe, root / "oracle" / "_ref" / "mclics_ref_gpu")
    monkeypatch.setattr(bench, "ROOT", str(root))
    monkeypatch.setattr(bench, "REFERENCE_GPU_SWEEPS", dict(bench.REFERENCE_GPU_SWEEPS, c4=(10, 20)))
    r, why = bench.reference_gpu(1, "sm_100", "c4")
    assert why is None
    runs = [line.split() for line in log.read_text().splitlines()]
    assert len(runs) == 3 * 6 and all(x[0] == "thermalGPU" and x[4] == "128" for x in runs)
    assert sorted({float(x[3]) for x in runs}) == [0.3, 0.8, 1.12]
    assert [(int(x[1]), int(x[2])) for x in runs[:6]] == [(200, 1)] * 2 + [(200, 11)] * 2 + [(220, 1)] * 2
    assert r["sites"] == 3 * 128 ** 3 and len(r["runs_s"]) == 3
    for name in ("c3", "c5"):
        r, why = bench.reference_gpu(1, "sm_100", name)
        assert r is None and "not timed" in why
