"""Replay parity: the reference's own CPU sweep (oracle/_ref, src/evolve.cpp:85-221) and the CUDA
reference-order kernel (MCL_SCHED_REF8) consume identical Philox draws from identical states, and must take
identical accept/reject decisions. The device state is re-synchronised from the reference before every sweep.

Tolerance: a decision may differ only when its random number lies within 1e-5 of exp(-dE/T) (device sinf/cosf/
expf may differ from glibc's by an ulp), or when a neighbour's decision did (its trial then sees another
neighbour). Directors of agreeing sites must match within 2e-6 and ang_var exactly."""
import numpy as np
import pytest

from helpers import M, O, engine_from_replay, explained_mismatches
from test_oracle_pin import CASES, SEED

GEOM = {"ll_bulk": "bulk", "ghrl_slab": "slab", "ghrl_chiral_homeo": "slab", "pear_field": "bulk",
        "sphere_rpt": "sphere", "slab_rp_fg": "slab", "t0": "bulk"}
TOL = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_ref8_kernel_replays_reference(name, tmp_path):
    assert O.ref_available(), "oracle/_ref must be built (make -C oracle)"
    n_sw = 6
    d = O.run_ref_replay(CASES[name], n_sw, SEED, str(tmp_path))
    m = O.model_from_replay(d)
    L = O.lattice_from_replay(d)
    e = engine_from_replay(d, GEOM[name], SEED, M.SCHED_REF8)
    e.record_decisions(True)
    valid = d["pt"] != 0
    total_near = 0
    for t, s in enumerate(d["sweeps"]):
        nxt = d["sweeps"][t + 1]["ni"] if t + 1 < n_sw else d["final"]
        e.upload(0, s["ni"])
        e.set_ang_var(s["ang_var"], 0)
        e.set_sweep_counter(t)
        e.sweeps(1)
        got = e.download(0)
        dec = e.decisions(0) & 3
        ni = s["ni"].copy()
        _, av, odec, margin = O.sweep(m, L, ni, d["T"], s["ang_var"], SEED, t, O.SCHED_REF8, True)
        assert np.array_equal(ni.view(np.uint32), nxt.view(np.uint32))  # oracle == reference
        mism = (dec != (odec & 3)) & valid
        hard, near = explained_mismatches(mism, margin, d["nx"], d["ny"], d["nz"], d["periodic"], TOL)
        total_near += near
        assert not hard, "sweep %d: unexplained decision mismatches at sites %s" % (t, hard[:10])
        agree = np.repeat(~mism, 3)
        assert np.max(np.abs(got[agree] - nxt[agree]), initial=0) <= 2e-6
        if not mism.any():
            assert e.ang_var(0) == s["ang_var_after"]
    assert total_near <= 2
