"""Pins the CPU oracle (oracle/mc_oracle.c) to the reference itself.

The reference's own CPU sources are compiled here with the GSL shim (oracle/Makefile -> oracle/_ref); the
replay driver runs the reference's EvolveN::Monte_Carlo_Step (src/evolve.cpp:85-221) on the Philox draws the
oracle uses, and the oracle must reproduce every sweep bit for bit: directors, ang_var and
energy_calculator (src/evolve.cpp:33-75). Also the Philox4x32-10 known-answer vectors of Random123 and the
reference's known-answer energies (tests/run_checks.py:156-204)."""
import numpy as np
import pytest

from helpers import O

SEED = 0xABCDEF12345

CASES = {
    "ll_bulk": "Nx 8\nNy 6\nNz 10\ngeometry bulk\nxbound periodic\nybound periodic\nzbound periodic\npotential ll\n"
               "A 1\nevol thermal\nTi 1.1\nTf 1.1\ndT -0.1\nic random\nseed 3\n",
    "ghrl_slab": "Nx 16\nNy 16\nNz 12\ngeometry slab\nxbound periodic\nybound periodic\npotential ghrl\nk11 1.48\n"
                 "k22 1\nk33 2.28\nanchoring_type 0 rp_ghrl\nanchoring_type 1 fg_ghrl\nW 0 1\nW 1 1\ntheta_s 0 90\n"
                 "phi_s 0 30\nevol thermal\nTi 0.5\nTf 0.5\ndT -0.1\nic random\nseed 6\n",
    "ghrl_chiral_homeo": "Nx 8\nNy 8\nNz 6\ngeometry slab\nxbound periodic\nybound free\npotential ghrl\nk11 1\n"
                         "k22 0.5\nk33 1.5\np0 12\nanchoring_type 0 homeotropic_ghrl\nW 0 1.5\n"
                         "anchoring_type 1 homeotropic\nW 1 1.5\nevol thermal\nTi 0.8\nTf 0.8\ndT -0.1\n"
                         "ic random\nseed 7\n",
    "pear_field": "Nx 6\nNy 6\nNz 8\ngeometry bulk\nxbound free\nybound free\nzbound periodic\npotential pear\n"
                  "A 1.5\nB1 0.09\nC 0.3\nelecP 0.5\nelecA 0.2\nelecX 0\nelecY 1\nelecZ 1\nevol thermal\nTi 0.4\n"
                  "Tf 0.4\ndT -0.1\nic random\nseed 2\n",
    "sphere_rpt": "Nx 11\nNy 11\nNz 11\ngeometry sphere\npotential ll\nanchoring_type 0 rp_tangent\nW 0 1.2\n"
                  "theta_s 0 30\nphi_s 0 20\nevol thermal\nTi 0.6\nTf 0.6\ndT -0.1\nic random\nseed 4\n",
    "slab_rp_fg": "Nx 8\nNy 8\nNz 7\ngeometry slab\nxbound periodic\nybound free\npotential ll\nanchoring_type 0 rp\n"
                  "theta_s 0 60\nphi_s 0 10\nW 0 0.8\nanchoring_type 1 fg\nW 1 0.7\nevol thermal\nTi 0.9\nTf 0.9\n"
                  "dT -0.1\nic random\nseed 5\n",
    "t0": "Nx 6\nNy 6\nNz 6\ngeometry bulk\nxbound periodic\nybound periodic\nzbound periodic\npotential ll\n"
          "evol thermal\nTi 0\nTf 0\ndT -0.1\nic random\nseed 8\n",
}


def test_philox_known_answers():
    # Random123 kat_vectors, philox4x32_10
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert O.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_reference_bit_for_bit(name, tmp_path):
    d = O.run_ref_replay(CASES[name], 5, SEED, str(tmp_path))
    m = O.model_from_replay(d)
    L = O.lattice_from_replay(d)
    for t, s in enumerate(d["sweeps"]):
        ni = s["ni"].copy()
        nxt = d["sweeps"][t + 1]["ni"] if t + 1 < len(d["sweeps"]) else d["final"]
        _, av, _, _ = O.sweep(m, L, ni, d["T"], s["ang_var"], SEED, t, O.SCHED_REF8)
        assert np.array_equal(ni.view(np.uint32), nxt.view(np.uint32)), "sweep %d directors differ" % t
        assert av == s["ang_var_after"]
        assert O.energy_ref(m, L, ni) == s["E_after"]
        assert len(O.ref8_stream(m, L, SEED, t)) == s["n_draws"]


def _uniform_z(n):
    ni = np.zeros(3 * n, np.float32)
    ni[2::3] = 1
    return ni


def test_known_answer_energies():
    """Ground-state energies of tests/run_checks.py:156-204, plus the uniform GHRL 1:0.5:1.5 and C2 slab."""
    L = O.Lat(8, 8, 8)
    ni = _uniform_z(L.n)
    assert O.energy_ref(O.make_model("ll", A=1), L, ni) == -9.0
    ghrl_eq = O.ghrl_coefficients(1, 1, 1)
    assert abs(O.energy_ref(O.make_model("ghrl", ghrl=ghrl_eq), L, ni) + 6.0) < 1e-5
    assert abs(O.energy_ref(O.make_model("pear", A=1.5, B1=0.09, C=0.3), L, ni) - 6 * (-1.5 - 0.09)) < 1e-5
    m = O.make_model("ll", field_dir=(0, 0, 1), elecA=0.5)
    assert abs(O.energy_ref(m, L, ni) + 9.5) < 1e-5
    c2 = O.ghrl_coefficients(1, 0.5, 1.5)
    np.testing.assert_allclose(c2, (1.0, -2.25, -1.0, -0.25, 0.0), rtol=1e-6)
    assert abs(O.energy_ref(O.make_model("ghrl", ghrl=c2), L, ni) + 9.0) < 1e-5
    # slab 8x8x6, x/y periodic, homeotropic W = 1 on both plates
    nz = 6
    pt = np.ones(8 * 8 * nz, np.int32)
    ns = np.zeros(3 * pt.size, np.float32)
    pt[:64] = 2
    ns[2:3 * 64:3] = -1
    pt[-64:] = 3
    ns[3 * (pt.size - 64) + 2::3] = 1
    Ls = O.Lat(8, 8, nz, (1, 1, 0), pt, ns)
    ms = O.make_model("ll", surfaces=[("homeotropic", 1, 0, 0), ("homeotropic", 1, 0, 0)])
    assert abs(O.energy_ref(ms, Ls, _uniform_z(Ls.n)) - (-1.5 * (256 * 6 + 128 * 5) - 128) / 384) < 1e-4


def test_oracle_eigen_and_q():
    rng = np.random.default_rng(0)
    v = rng.normal(size=(500, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    q = np.einsum("ni,nj->ij", v, v) * 1.5 / 500 - 0.5 * np.eye(3)
    s, vec = O.largest_eigen([q[0, 0], q[0, 1], q[0, 2], q[1, 1], q[1, 2], q[2, 2]])
    w, V = np.linalg.eigh(q)
    assert abs(s - w[-1]) < 1e-13
    assert abs(abs(vec @ V[:, -1]) - 1) < 1e-10
