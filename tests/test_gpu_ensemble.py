"""Ensemble parity with the reference: for each golden case (tests/golden/ensemble_<case>.json, made by
tests/golden/make_ensemble.py from the reference's own CPU program) this build's driver runs the same input file for
the same seeds on the GPU. The two are different Markov chains (two-colour vs eight-sublattice order, Philox vs
the reference's generators) with the same equilibrium, so at every scan point the seed means of every po.dat column
(S, varS, E, varE, and P, dtheta, divn for pear) must agree within 3 standard errors, the two ensembles' errors
combined, and the mean of z^2 over a case's comparisons must stay below 2.1. Cases: LL 16^3 thermal scan; the C1
scan itself (32^3 LL, 11 temperatures); C2's physics (GHRL 1 : 0.5 : 1.5 slab, homeotropic W = 1.5); C5's physics
(pear slab, planar anchoring, dipolar field, flip move; 64 seeds of the reference, 128 here)."""
import json
import os

import numpy as np
import pytest

from helpers import M, input_text, read_po

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["ll16", "c1_scan", "ghrl_slab", "pear_field"]
# seeds run here per seed of the fixture: the two ensembles are independent (their standard errors add), and this
# side is cheap, so the slow case's comparison is limited by the reference program's own seeds
SEEDS_HERE = {"pear_field": 2}


def run_ours(tmp_path, params, seed, columns):
    d = os.path.join(str(tmp_path), "seed%d" % seed)
    os.makedirs(d)
    with open(os.path.join(d, "input.txt"), "w") as f:
        f.write(input_text([tuple(p) for p in params] + [("seed", seed)]))
    cwd = os.getcwd()
    os.chdir(d)
    try:
        M.run_input_file("input.txt")
    finally:
        os.chdir(cwd)
    header, rows = read_po(d)
    assert header == columns
    return [[r[k] for k in columns] for r in rows]


@pytest.mark.parametrize("case", CASES)
def test_ensemble_matches_reference(tmp_path, case):
    with open(os.path.join(GOLDEN, "ensemble_%s.json" % case)) as f:
        g = json.load(f)
    cols = g["po_header"]
    ref = np.array([g["rows"][str(s)] for s in g["seeds"]])
    seeds = g["seeds"] + [10000 + s for s in range(len(g["seeds"]) * (SEEDS_HERE.get(case, 1) - 1))]
    ours = np.array([run_ours(tmp_path, g["params"], s, cols) for s in seeds])
    assert ours.shape[1:] == ref.shape[1:]
    assert np.allclose(ours[0, :, 0], ref[0, :, 0])  # the same scan points, in the same order
    report = []
    for t in range(ref.shape[1]):
        for c in range(1, len(cols)):
            a, b = ref[:, t, c], ours[:, t, c]
            se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
            z = (b.mean() - a.mean()) / se if se > 0 else 0.0
            report.append((cols[0], ref[0, t, 0], cols[c], a.mean(), b.mean(), se, z))
    for r in report:
        print("%s=%g %-6s reference %.6g  this build %.6g  se %.3g  z %+.2f" % r)
    worst = max(abs(r[6]) for r in report)
    print("%s: %d comparisons, largest |z| %.2f" % (case, len(report), worst))
    bad = [r for r in report if abs(r[6]) > 3.0]
    assert not bad, "\n".join("%s=%g %s ref %.6g ours %.6g se %.3g z %.2f" % r for r in bad)
    # and as a whole: the mean of z^2 over a case's comparisons (1 without a difference; 2.1 lies in the 1-2 % tail
    # of chi-square / k for the 8 to 48 comparisons of these cases, or beyond it)
    chi = float(np.mean([r[6] ** 2 for r in report]))
    print("%s: mean z^2 %.2f" % (case, chi))
    assert chi < 2.1, chi
