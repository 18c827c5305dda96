"""Generates tests/golden/ensemble_ll16.json, the golden ensemble of tests/test_gpu_ensemble.py: the reference's own
CPU program (oracle/_ref/mclics_ref, built by oracle/Makefile from the reference sources with the GSL stand-in)
run on a thermal scan of a 16^3 periodic LL lattice for 12 seeds; per seed and temperature the po.dat row
(T, S, varS, E, varE).

    python tests/golden/make_ensemble.py      # needs oracle/_ref/mclics_ref (built where the reference is)
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
OUT = os.path.join(HERE, "ensemble_ll16.json")

PARAMS = [("Nx", 16), ("Ny", 16), ("Nz", 16), ("geometry", "bulk"), ("xbound", "periodic"), ("ybound", "periodic"),
          ("zbound", "periodic"), ("potential", "ll"), ("A", 1), ("evol", "thermal"), ("Ti", 1.3), ("Tf", 0.9),
          ("dT", -0.2), ("MCT", 400), ("MCS", 1000), ("ic", "random")]
SEEDS = list(range(1, 13))


def input_text(seed):
    return "".join("%s %s\n" % kv for kv in PARAMS + [("seed", seed)])


def read_po(path):
    with open(path) as f:
        lines = [l.split() for l in f if l.strip()]
    header = lines[0]
    return [[float(v) for v in l] for l in lines[1:]], header


def main():
    if not os.path.exists(EXE):
        sys.exit("oracle/_ref/mclics_ref is not built (make -C oracle)")
    rows, header = {}, None
    t0 = time.time()
    for seed in SEEDS:
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "input.txt"), "w") as f:
                f.write(input_text(seed))
            subprocess.run([EXE, "input.txt"], cwd=d, check=True, capture_output=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1)))
            rows[str(seed)], header = read_po(os.path.join(d, "po.dat"))
    doc = {"generator": "oracle/_ref/mclics_ref (reference CPU sources, GSL stand-in RNG)",
           "script": "tests/golden/make_ensemble.py", "params": PARAMS, "seeds": SEEDS, "po_header": header,
           "rows": rows, "seconds": round(time.time() - t0, 1)}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT, "in %.1f s" % doc["seconds"])


if __name__ == "__main__":
    main()
