"""Ensemble parity with the reference: the same thermal scan (16^3 periodic LL, T = 1.3, 1.1, 0.9, MCT 400, MCS 1000,
random initial condition) for the same 12 seeds, run by the reference's own CPU program (the golden fixture,
tests/golden/ensemble_ll16.json, made by tests/golden/make_ensemble.py) and by this build's driver on the GPU. The
two are different Markov chains (two-colour vs eight-sublattice order, Philox vs the reference's generators) with
the same equilibrium, so for every temperature the seed means of S, varS, E and varE must agree within 3 standard
errors (the two ensembles' errors combined)."""
import json
import os

import numpy as np
import pytest

from helpers import M, input_text, read_po

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ensemble_ll16.json")


def run_ours(tmp_path, params, seed):
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
    return [[r[k] for k in ("T", "S", "varS", "E", "varE")] for r in rows]


def test_ensemble_matches_reference(tmp_path):
    with open(GOLDEN) as f:
        g = json.load(f)
    assert g["po_header"] == ["T", "S", "varS", "E", "varE"]
    ref = np.array([g["rows"][str(s)] for s in g["seeds"]])
    ours = np.array([run_ours(tmp_path, g["params"], s) for s in g["seeds"]])
    assert ours.shape == ref.shape
    assert np.allclose(ours[:, :, 0], ref[:, :, 0])  # the same temperatures, in the same order
    n = len(g["seeds"])
    report = []
    for t in range(ref.shape[1]):
        for c, name in enumerate(["S", "varS", "E", "varE"], start=1):
            a, b = ref[:, t, c], ours[:, t, c]
            se = np.sqrt(a.var(ddof=1) / n + b.var(ddof=1) / n)
            z = (b.mean() - a.mean()) / se if se > 0 else 0.0
            report.append((ref[0, t, 0], name, a.mean(), b.mean(), se, z))
    for r in report:
        print("T=%g %-4s reference %.6g  this build %.6g  se %.3g  z %+.2f" % r)
    bad = [r for r in report if abs(r[5]) > 3.0]
    assert not bad, "\n".join("T=%g %s ref %.6g ours %.6g se %.3g z %.2f" % r for r in report)
