"""Generates the golden ensembles of tests/test_gpu_ensemble.py: the reference's own CPU program
(oracle/_ref/mclics_ref, built by oracle/Makefile from the reference sources with the GSL stand-in) run on each
case below for 16 seeds; per seed, every po.dat row (the scanned value, S, varS, E, varE and the extra columns).

    python tests/golden/make_ensemble.py [case ...]   # needs oracle/_ref/mclics_ref (built where the reference is)

Cases (one file tests/golden/ensemble_<case>.json each):
  ll16        16^3 periodic LL, thermal scan T = 1.3, 1.1, 0.9 from a random start.
  c1_scan     the C1 configuration as stated: 32^3 periodic LL, thermal scan Ti = 1.2 -> Tf = 1.0 (dT = -0.02,
              11 temperatures), MCT 500, MCS 200, random start.
  ghrl_slab   C2's physics on a 24 x 24 x 16 slab: GHRL with K11:K22:K33 = 1 : 0.5 : 1.5, homeotropic anchoring
              W = 1.5 on both plates, x and y periodic, T = 0.8 and 0.6, start along z.
  pear_field  C5's physics on a 16 x 16 x 8 slab: pear (A, B1, C at the reference defaults), planar degenerate
              anchoring (fg) W = 1 on both plates, dipolar field along z (elecP = 1) at E = 0 and E = 2, the flip
              move on, T = 0.5, random start; at zero field polar domains coarsen over thousands of sweeps, hence
              MCT 8000, MCS 4000 and 64 seeds.
"""
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "mclics_ref")

SEEDS = list(range(1, 17))
PERIODIC = [("xbound", "periodic"), ("ybound", "periodic"), ("zbound", "periodic")]
CASES = {
    "ll16": [("Nx", 16), ("Ny", 16), ("Nz", 16), ("geometry", "bulk")] + PERIODIC + [
        ("potential", "ll"), ("A", 1), ("evol", "thermal"), ("Ti", 1.3), ("Tf", 0.9), ("dT", -0.2), ("MCT", 1500),
        ("MCS", 1000), ("ic", "random")],
    "c1_scan": [("Nx", 32), ("Ny", 32), ("Nz", 32), ("geometry", "bulk")] + PERIODIC + [
        ("potential", "ll"), ("A", 1.0), ("evol", "thermal"), ("Ti", 1.2), ("Tf", 1.0), ("dT", -0.02), ("MCT", 500),
        ("MCS", 200), ("ic", "random")],
    "ghrl_slab": [("Nx", 24), ("Ny", 24), ("Nz", 16), ("geometry", "slab"), ("xbound", "periodic"),
                  ("ybound", "periodic"), ("potential", "ghrl"), ("k11", 1), ("k22", 0.5), ("k33", 1.5),
                  ("anchoring_type 0", "homeotropic"), ("W 0", 1.5), ("anchoring_type 1", "homeotropic"),
                  ("W 1", 1.5), ("evol", "thermal"), ("Ti", 0.8), ("Tf", 0.6), ("dT", -0.2), ("MCT", 2000),
                  ("MCS", 2000), ("ic", "homogeneous"), ("theta_0", 0), ("phi_0", 0)],
    "pear_field": [("Nx", 16), ("Ny", 16), ("Nz", 8), ("geometry", "slab"), ("xbound", "periodic"),
                   ("ybound", "periodic"), ("potential", "pear"), ("A", 1.0), ("B1", 0.04), ("C", 0.3),
                   ("anchoring_type 0", "fg"), ("W 0", 1.0), ("anchoring_type 1", "fg"), ("W 1", 1.0),
                   ("elecX", 0), ("elecY", 0), ("elecZ", 1), ("elecP", 1.0), ("evol", "electric"), ("Ti", 0.5),
                   ("Ei", 0.0), ("Ef", 2.0), ("dE", 2.0), ("MCT", 8000), ("MCS", 4000), ("ic", "random")],
}
SEED_COUNT = {"pear_field": 64}  # the others: 16


def input_text(params, seed):
    return "".join("%s %s\n" % kv for kv in params + [("seed", seed)])


def read_po(path):
    with open(path) as f:
        lines = [l.split() for l in f if l.strip()]
    return [[float(v) for v in l] for l in lines[1:]], lines[0]


def make(case):
    params = CASES[case]
    seeds = list(range(1, SEED_COUNT.get(case, len(SEEDS)) + 1))
    rows, header = {}, None
    t0 = time.time()
    for seed in seeds:
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "input.txt"), "w") as f:
                f.write(input_text(params, seed))
            subprocess.run([EXE, "input.txt"], cwd=d, check=True, capture_output=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)))
            rows[str(seed)], header = read_po(os.path.join(d, "po.dat"))
    doc = {"case": case, "generator": "oracle/_ref/mclics_ref (reference CPU sources, GSL stand-in RNG)",
           "script": "tests/golden/make_ensemble.py", "params": params, "seeds": seeds, "po_header": header,
           "rows": rows, "seconds": round(time.time() - t0, 1)}
    out = os.path.join(HERE, "ensemble_%s.json" % case)
    with open(out, "w") as f:
        json.dump(doc, f, indent=0)
    print("wrote", out, "in %.1f s" % doc["seconds"])


def main():
    if not os.path.exists(EXE):
        sys.exit("oracle/_ref/mclics_ref is not built (make -C oracle REF=<reference source tree>)")
    for case in sys.argv[1:] or list(CASES):
        make(case)


if __name__ == "__main__":
    main()
