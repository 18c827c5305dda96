"""Shared helpers of the test suite: reference-style input files, replay-dump -> engine conversion."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import mclics_b200 as M  # noqa: E402
from oracle import oracle as O  # noqa: E402


def input_text(params):
    """params: dict or list of (name, value) -> McLics input file text."""
    items = params.items() if isinstance(params, dict) else params
    return "".join("%s %s\n" % (k, v) for k, v in items)


def base(**kw):
    """Small periodic bulk at T = 0 from the uniform state along z, one measurement sweep (the reference's
    tests/run_checks.py `base()` case, restated)."""
    p = dict(Nx=8, Ny=8, Nz=8, geometry="bulk", xbound="periodic", ybound="periodic", zbound="periodic",
             potential="ll", A=1, evol="thermalGPU", Ti=0, Tf=0, dT=-0.1, MCT=0, MCS=1, ic="homogeneous",
             theta_0=0, phi_0=0, seed=1)
    p.update(kw)
    return p


def plus(params, *lines):
    return list(params.items()) + [tuple(l.split(None, 1)) for l in lines]


def read_po(d):
    with open(os.path.join(d, "po.dat")) as f:
        lines = [l.split() for l in f if l.strip()]
    header = lines[0]
    rows = [dict(zip(header, map(float, l))) for l in lines[1:]]
    return header, rows


GEOM_OF = {"bulk": 0, "slab": 1, "sphere": 2, "custom": 3}


def engine_from_replay(d, geometry, seed, schedule):
    """Engine with the exact model and lattice of a reference replay dump (no re-normalisation of the field)."""
    m = M.CModel()
    m.potential = d["potential"]
    m.A, m.B1, m.C = d["A"], d["B1"], d["C"]
    m.ghrl_lambda, m.ghrl_mu, m.ghrl_nu, m.ghrl_rho, m.ghrl_sigma = (d["lambda"], d["mu"], d["nu"], d["rho"],
                                                                     d["sigma"])
    m.field_dir[:] = [d["elecX"], d["elecY"], d["elecZ"]]
    m.elecA, m.elecP = d["elecA"], d["elecP"]
    m.flip_move = d["flip_move"]
    m.n_surfaces = len(d["surfaces"])
    for s, (t, W, th, ph) in enumerate(d["surfaces"]):
        m.anch_type[s], m.anch_W[s], m.anch_theta[s], m.anch_phi[s] = t, W, th, ph
    r = M.Replica(d["nx"], d["ny"], d["nz"], geometry, d["periodic"], T=d["T"], elecE=d["elecE"], seed=seed)
    e = M.Engine(m, [r], schedule)
    if GEOM_OF[geometry] >= 2:
        e.set_geometry(0, d["pt"], d["ns"])
    return e


def neighbours(idx, nx, ny, nz, periodic):
    i, j, k = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    out = []
    for a, (c, n) in enumerate(((i, nx), (j, ny), (k, nz))):
        for s in (1, -1):
            v = c + s
            if periodic[a]:
                v %= n
            elif v < 0 or v >= n:
                continue
            q = [i, j, k]
            q[a] = v
            out.append(q[0] + nx * (q[1] + ny * q[2]))
    return out


def explained_mismatches(mismatch, margin, nx, ny, nz, periodic, tol):
    """Decision mismatches that are not explained by a near-threshold decision at the site itself or at one of
    its neighbours (which changes the neighbour's later trial)."""
    near = set(np.nonzero(mismatch & (margin < tol))[0].tolist())
    hard = []
    for idx in np.nonzero(mismatch)[0].tolist():
        if idx in near:
            continue
        if any(q in near for q in neighbours(idx, nx, ny, nz, periodic)):
            continue
        hard.append(idx)
    return hard, len(near)
