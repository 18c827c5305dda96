"""The compiled drop-in: the reference's own program (its main.cpp, simulator.cpp, io.cpp, geometry and IC code)
with this library behind its *GPU modes (mclics_b200/adapter/evolve_ngpu_b200.cu, built by
mclics_b200/adapter/Makefile into mclics_b200/adapter/_build/mclics_dropin). It runs the same input files as the
reference's own CPU program (oracle/_ref/mclics_ref) in the matching CPU mode:
  * at T = 0 from a ground state no trial move is accepted, so po.dat, ic.csv and every snapshot must be
    byte-identical between the two programs;
  * at T > 0 the two are different Markov chains: the file names, headers, column sets, scan points and ic.csv
    (the reference's own initial-condition code in both) must be identical, the values physically consistent;
  * input errors are reported by the reference's own validation, with the same exit status and message."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "mclics_b200", "adapter", "_build", "mclics_dropin")
REFCPU = os.path.join(ROOT, "oracle", "_ref", "mclics_ref")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFCPU)),
                                 reason="the drop-in and the reference CPU program are built where the reference "
                                        "sources are (make -C mclics_b200/adapter REF=..., make -C oracle REF=...)")]


def base(**kw):
    p = dict(Nx=8, Ny=8, Nz=8, geometry="bulk", xbound="periodic", ybound="periodic", zbound="periodic",
             potential="ll", A=1, evol="thermal", Ti=0, Tf=0, dT=-0.1, MCT=0, MCS=1, ic="homogeneous", theta_0=0,
             phi_0=0, seed=1)
    p.update(kw)
    return p


def run(program, folder, params, gpu, extra_lines=()):
    os.makedirs(folder)
    lines = ["%s %s" % (k, (v + "GPU") if (k == "evol" and gpu) else v) for k, v in params.items()]
    with open(os.path.join(folder, "input.txt"), "w") as f:
        f.write("\n".join(lines + list(extra_lines)) + "\n")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run([program, "input.txt"], cwd=folder, env=env, capture_output=True, text=True, timeout=600)
    return p


def outputs(folder):
    return sorted(f for f in os.listdir(folder) if f == "po.dat" or f == "ic.csv" or f.startswith("director_field_"))


def read(folder, name):
    with open(os.path.join(folder, name)) as f:
        return f.read()


def both(tmp_path, params, extra_lines=()):
    a = run(REFCPU, os.path.join(str(tmp_path), "reference"), params, False, extra_lines)
    b = run(DROPIN, os.path.join(str(tmp_path), "dropin"), params, True, extra_lines)
    return a, b, os.path.join(str(tmp_path), "reference"), os.path.join(str(tmp_path), "dropin")


GROUND = [
    ("ll", base(), ()),
    ("ghrl_equal_k", base(potential="ghrl", k11=1, k22=1, k33=1), ()),
    ("pear", base(potential="pear", A=1.5, B1=0.09, C=0.3), ()),
    ("slab_homeotropic_ghrl_c2", base(Nx=8, Ny=8, Nz=6, geometry="slab", potential="ghrl", k11=1, k22=0.5, k33=1.5),
     ("anchoring_type 0 homeotropic", "W 0 1.5", "anchoring_type 1 homeotropic", "W 1 1.5")),
    ("field", base(elecA=0.5, elecX=0, elecY=0, elecZ=2), ()),
    ("step_blocks", base(evol="step", fn=2, first_file_number=3), ()),
]


@pytest.mark.parametrize("name,params,extra", GROUND, ids=[g[0] for g in GROUND])
def test_ground_states_byte_identical(tmp_path, name, params, extra):
    a, b, da, db = both(tmp_path, params, extra)
    assert a.returncode == 0, a.stderr
    assert b.returncode == 0, b.stderr
    assert outputs(da) == outputs(db)
    for f in outputs(da):
        assert read(da, f) == read(db, f), f


def test_electric_scan_ground_states(tmp_path):
    """A field scan from the ground state: the snapshots and ic.csv are byte-identical; in po.dat the energies at
    field 0.2 and 0.4 (-9.012, -9.048 per site) are not exact floats, so varE = <E^2> - <E>^2 is rounding noise of
    order 1e-6 on either side and is compared to that level, the other columns as printed."""
    a, b, da, db = both(tmp_path, base(evol="electric", Ei=0, Ef=0.4, dE=0.2, elecA=0.3, elecZ=1))
    assert a.returncode == 0 and b.returncode == 0, a.stderr + b.stderr
    assert outputs(da) == outputs(db)
    for f in outputs(da):
        if f != "po.dat":
            assert read(da, f) == read(db, f), f
    pa, pb = read(da, "po.dat").splitlines(), read(db, "po.dat").splitlines()
    assert pa[0] == pb[0] == "field S varS E varE" and len(pa) == len(pb) == 4
    for la, lb in zip(pa[1:], pb[1:]):
        ra, rb = la.split(), lb.split()
        assert ra[:4] == rb[:4], (la, lb)
        assert abs(float(ra[4]) - float(rb[4])) < 1e-5, (la, lb)


def test_thermal_scan_same_files_and_format(tmp_path):
    p = base(Nx=10, Ny=8, Nz=6, Ti=1.2, Tf=1.0, dT=-0.1, MCT=20, MCS=30, ic="random", seed=4)
    a, b, da, db = both(tmp_path, p)
    assert a.returncode == 0 and b.returncode == 0, a.stderr + b.stderr
    assert outputs(da) == outputs(db)
    assert read(da, "ic.csv") == read(db, "ic.csv")  # the reference's own random initial condition, same seed
    pa, pb = read(da, "po.dat").splitlines(), read(db, "po.dat").splitlines()
    assert pa[0] == pb[0] == "T S varS E varE"
    assert len(pa) == len(pb) == 4
    for la, lb in zip(pa[1:], pb[1:]):
        ra, rb = la.split(), lb.split()
        assert ra[0] == rb[0] and len(ra) == len(rb) == 5
        E, S = float(rb[3]), float(rb[1])
        assert -9.0 < E < 0.0 and 0.0 < S < 1.0
    for f in outputs(da):
        if f.startswith("director_field_"):
            sa, sb = read(da, f).splitlines(), read(db, f).splitlines()
            assert sa[0] == sb[0] == "x,y,z,nx,ny,nz,S,pt"
            assert len(sa) == len(sb) == 1 + 10 * 8 * 6
            assert [l.split(",")[:3] + l.split(",")[7:] for l in sa[1:]] == \
                [l.split(",")[:3] + l.split(",")[7:] for l in sb[1:]]


def test_pear_sphere_extra_columns(tmp_path):
    p = base(Nx=12, Ny=12, Nz=12, geometry="sphere", potential="pear", A=1.5, B1=0.09, C=0.3, Ti=0.3, Tf=0.3,
             MCT=5, MCS=5, ic="random")
    a, b, da, db = both(tmp_path, p, ("anchoring_type 0 homeotropic", "W 0 1.5"))
    assert a.returncode == 0 and b.returncode == 0, a.stderr + b.stderr
    ha, hb = read(da, "po.dat").splitlines()[0], read(db, "po.dat").splitlines()[0]
    assert ha == hb == "T S varS E varE P dtheta divn Sr_sph Pr_sph"
    assert read(da, "ic.csv") == read(db, "ic.csv")


ERRORS = [
    ("odd_periodic", base(Nx=5), (), "even"),
    ("wrong_dT", base(Ti=0.5, Tf=1.0, dT=-0.1), (), "dT"),
    ("unknown_parameter", base(), ("Tff 0.1",), "Unknown parameter"),
    ("missing_anchoring", base(Nz=6, geometry="slab"), ("anchoring_type 0 homeotropic", "W 0 1"), "anchoring_type 1"),
]


@pytest.mark.parametrize("name,params,extra,text", ERRORS, ids=[e[0] for e in ERRORS])
def test_input_errors_as_the_reference(tmp_path, name, params, extra, text):
    a, b, _, _ = both(tmp_path, params, extra)
    assert a.returncode != 0 and b.returncode == a.returncode
    assert text in a.stderr and text in b.stderr
