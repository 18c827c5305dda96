"""The whole-program path (mcl_run_input_file): known answers of the reference's tests/run_checks.py:111-347
(ground-state energies, sweep points and snapshot names, modes, snapshot read back as ic_file), on the GPU."""
import math
import os
import shutil

import pytest

from helpers import M, base, input_text, plus, read_po


def run(tmp_path, params, files=None, name="run"):
    d = os.path.join(str(tmp_path), name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "input.txt"), "w") as f:
        f.write(input_text(params))
    for k, v in (files or {}).items():
        with open(os.path.join(d, k), "w") as f:
            f.write(v)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        M.run_input_file("input.txt")
    finally:
        os.chdir(cwd)
    return d


def snapshots(d):
    return sorted(f for f in os.listdir(d) if f.startswith("director_field_"))


@pytest.mark.gpu
def test_ground_state_ll(tmp_path):
    _, rows = read_po(run(tmp_path, base()))
    assert abs(rows[0]["E"] + 9.0) <= 1e-4 and abs(rows[0]["S"] - 1.0) <= 1e-5 and abs(rows[0]["varE"]) <= 1e-8


@pytest.mark.gpu
def test_ground_state_ghrl_equal_k(tmp_path):
    _, rows = read_po(run(tmp_path, base(potential="ghrl", k11=1, k22=1, k33=1)))
    assert abs(rows[0]["E"] + 6.0) <= 1e-4


@pytest.mark.gpu
def test_ground_state_pear(tmp_path):
    _, rows = read_po(run(tmp_path, base(potential="pear", A=1.5, B1=0.09, C=0.3)))
    assert abs(rows[0]["E"] - 6 * (-1.5 - 0.09)) <= 1e-4
    assert abs(rows[0]["P"] - 1.0) <= 1e-5


@pytest.mark.gpu
def test_ground_state_slab_homeotropic(tmp_path):
    p = plus(base(Nz=6, geometry="slab"), "anchoring_type 0 homeotropic", "W 0 1", "anchoring_type 1 homeotropic",
             "W 1 1")
    _, rows = read_po(run(tmp_path, p))
    assert abs(rows[0]["E"] - (-1.5 * (256 * 6 + 128 * 5) - 128) / 384) <= 1e-4


@pytest.mark.gpu
def test_ground_state_field(tmp_path):
    _, rows = read_po(run(tmp_path, base(elecA=0.5, elecX=0, elecY=0, elecZ=2)))
    assert abs(rows[0]["E"] + 9.5) <= 1e-4


@pytest.mark.gpu
def test_ground_state_c2_ghrl_slab(tmp_path):
    """C2's potential and anchoring on a uniform z state: 5 bonds of -1.5 and -1.5 W... per surface site."""
    p = plus(base(Nx=16, Ny=16, Nz=8, geometry="slab", potential="ghrl", k11=1, k22=0.5, k33=1.5),
             "anchoring_type 0 homeotropic", "W 0 1.5", "anchoring_type 1 homeotropic", "W 1 1.5")
    _, rows = read_po(run(tmp_path, p))
    n_plane = 256
    expect = (-1.5 * (n_plane * 8 * 6 - 2 * n_plane) - 1.5 * 2 * n_plane) / (n_plane * 8)
    assert abs(rows[0]["E"] - expect) <= 1e-4


def hedgehog_csv(n, sign=1):
    c = n // 2
    out = ["x,y,z,nx,ny,nz"]
    for k in range(n):
        for j in range(n):
            for i in range(n):
                v = (i - c, j - c, k - c)
                m = math.sqrt(sum(x * x for x in v))
                u = (0, 0, 1) if m == 0 else tuple(sign * x / m for x in v)
                out.append("%d,%d,%d,%.6f,%.6f,%.6f" % ((i, j, k) + u))
    return "\n".join(out) + "\n"


@pytest.mark.gpu
def test_hedgehog_radial_order(tmp_path):
    p = plus(base(Nx=21, Ny=21, Nz=21, geometry="sphere", potential="pear", A=1.5, B1=0.09, C=0.3, ic="ic_file",
                  ic_file="hedgehog.csv"), "anchoring_type 0 homeotropic", "W 0 1.5")
    header, rows = read_po(run(tmp_path, p, files={"hedgehog.csv": hedgehog_csv(21)}))
    for col in ("P", "dtheta", "divn", "Sr_sph", "Pr_sph"):
        assert col in header
    assert abs(rows[0]["Sr_sph"] - 1.0) <= 0.03
    assert abs(rows[0]["Pr_sph"] - 1.0) <= 0.03
    assert abs(rows[0]["divn"] - 0.275) <= 0.02


@pytest.mark.gpu
def test_columns_ll_sphere(tmp_path):
    p = plus(base(Nx=11, Ny=11, Nz=11, geometry="sphere", ic="random"), "anchoring_type 0 homeotropic", "W 0 1")
    header, _ = read_po(run(tmp_path, p))
    assert header == ["T", "S", "varS", "E", "varE", "Sr_sph"]


@pytest.mark.gpu
def test_thermal_sweep_points(tmp_path):
    d = run(tmp_path, base(Nx=4, Ny=4, Nz=4, Ti=1.0, Tf=0.5, dT=-0.1, ic="random"))
    _, rows = read_po(d)
    T = [r["T"] for r in rows]
    assert len(T) == 6 and all(abs(a - b) < 1e-6 for a, b in zip(T, [1.0, 0.9, 0.8, 0.7, 0.6, 0.5]))
    assert snapshots(d) == sorted("director_field_%d.csv" % v for v in (100, 90, 80, 70, 60, 50))


@pytest.mark.gpu
def test_thermal_fine_step_names(tmp_path):
    d = run(tmp_path, base(Nx=4, Ny=4, Nz=4, Ti=1.24, Tf=1.224, dT=-0.004, ic="random"))
    _, rows = read_po(d)
    assert len(rows) == 5
    assert snapshots(d) == sorted("director_field_%d.csv" % v for v in (1240, 1236, 1232, 1228, 1224))


@pytest.mark.gpu
def test_thermal_step_001_names(tmp_path):
    d = run(tmp_path, base(Nx=4, Ny=4, Nz=4, Ti=1.2, Tf=1.1, dT=-0.01, ic="random"))
    assert snapshots(d) == sorted("director_field_%d.csv" % v for v in range(110, 121))


@pytest.mark.gpu
def test_electric_sweep(tmp_path):
    d = run(tmp_path, base(Nx=4, Ny=4, Nz=4, evol="electricGPU", Ti=0.5, elecA=0.1, elecZ=1, Ei=0, Ef=1.2, dE=0.1,
                           ic="random"))
    header, rows = read_po(d)
    assert header[0] == "field"
    E = [r["field"] for r in rows]
    assert len(E) == 13 and abs(E[-1] - 1.2) < 1e-6


@pytest.mark.gpu
def test_step_blocks(tmp_path):
    d = run(tmp_path, base(Nx=4, Ny=4, Nz=4, evol="stepGPU", Ti=0.5, fn=3, first_file_number=5, MCT=2, ic="random"))
    header, rows = read_po(d)
    assert header[0] == "ii" and [r["ii"] for r in rows] == [5, 6, 7]
    assert snapshots(d) == ["director_field_5.csv", "director_field_6.csv", "director_field_7.csv"]


@pytest.mark.gpu
def test_quench_relaxes(tmp_path):
    _, rows = read_po(run(tmp_path, base(evol="quenchGPU", Ti=2.0, Tf=0.5, MCT=50, MCQ=300, MCS=20, fn=1,
                                         ic="random")))
    assert rows[0]["S"] > 0.8


@pytest.mark.gpu
def test_snapshot_as_ic_file(tmp_path):
    d1 = run(tmp_path, base(Nx=6, Ny=6, Nz=6, Ti=0.3, Tf=0.3, MCT=5, ic="random"), name="a")
    snap = os.path.join(d1, "director_field_30.csv")
    d2 = os.path.join(str(tmp_path), "b")
    os.makedirs(d2)
    shutil.copy(snap, os.path.join(d2, "start.csv"))
    run(tmp_path, base(Nx=6, Ny=6, Nz=6, ic="ic_file", ic_file="start.csv"), name="b")

    def directors(path):
        with open(path) as f:
            next(f)
            return [tuple(round(float(x), 5) for x in l.split(",")[3:6]) for l in f]
    assert directors(snap) == directors(os.path.join(d2, "ic.csv"))


@pytest.mark.gpu
def test_same_seed_same_po(tmp_path):
    p = base(Nx=6, Ny=6, Nz=6, Ti=0.8, Tf=0.8, MCT=20, MCS=20, ic="random")
    a = run(tmp_path, p, name="a")
    b = run(tmp_path, p, name="b")
    p["seed"] = 2
    c = run(tmp_path, p, name="c")
    po = [open(os.path.join(x, "po.dat")).read() for x in (a, b, c)]
    assert po[0] == po[1] and po[0] != po[2]
