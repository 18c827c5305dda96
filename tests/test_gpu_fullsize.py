"""The benchmark lattice itself against the oracle: one sweep of the full 256^3 GHRL slab (K11 : K22 : K33 =
1 : 0.5 : 1.5, homeotropic W = 1.5 on both plates, x and y periodic, T = 0.8, seed 7) with the tile plan the
autotuner picks for it, compared with the oracle's two-colour sweep from the same state under the two-colour
criteria of the small cases: decisions identical except next to the acceptance threshold (or next to such a
site), directors of agreeing sites within 1e-5, FP64 observables of the swept state within the stated tolerances.
Three comparisons: from the (0, 0, 1) + 0.1 noise start, after 20 sweeps, and after 20 more with the plan the
colour passes use by default for non-flip models."""
import numpy as np
import pytest

from helpers import M, O, explained_mismatches

pytestmark = pytest.mark.gpu

NX = NY = NZ = 256
T = 0.8
SEED = 7
TOL = 3e-5
NEAR_PER_SITE = 2e-5  # near-threshold decisions allowed per site and sweep (FP32 / FMA energies, fast exp)


def slab_geometry():
    n = NX * NY * NZ
    pt = np.ones(n, np.int32)
    ns = np.zeros(3 * n, np.float32)
    plane = NX * NY
    pt[:plane] = 2
    ns[2:3 * plane:3] = -1
    pt[-plane:] = 3
    ns[3 * (n - plane) + 2::3] = 1
    return pt, ns


def z_noise(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-0.1, 0.1, size=(n, 3)).astype(np.float32)
    v[:, 2] += 1.0
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v.reshape(-1).astype(np.float32)


def compare_one_sweep(e, om, L, ni, av, t):
    """One measured engine sweep from ni (rotation amplitude av, sweep index t) against the oracle's."""
    e.upload(0, ni)
    e.set_ang_var(av, 0)
    e.set_sweep_counter(t)
    e.sweeps(1, measure=True)
    got = e.download(0)
    o = e.series(0)[-1]
    ref = ni.copy()
    acc, av_next, dec, margin = O.sweep(om, L, ref, T, av, SEED, t, O.SCHED_CHECKER2, True)
    moved_gpu = np.any(got.reshape(-1, 3) != ni.reshape(-1, 3), axis=1)
    moved_ref = np.any(ref.reshape(-1, 3) != ni.reshape(-1, 3), axis=1)
    # A rotation angle draw of exactly 1/2 (one site in 2^21: about 8 per sweep here) gives a zero rotation; both
    # sides accept it, and the renormalisation (reciprocal square root here, square root and division in the
    # oracle) may change the director by an ulp on one side only. A decision differs when the directors do.
    differ = np.abs(got - ref).reshape(-1, 3).max(axis=1) > 1e-5
    mism = (moved_gpu != moved_ref) & differ
    hard, near = explained_mismatches(mism, margin, NX, NY, NZ, L.c.periodic, TOL)
    n = NX * NY * NZ
    print("sweep %d: %d of %d sites moved, %d decisions differ (%d next to the threshold), %d zero rotations"
          % (t, int(moved_ref.sum()), n, int(mism.sum()), near, int(((moved_gpu != moved_ref) & ~differ).sum())))
    assert not hard, "sweep %d: unexplained mismatches %s" % (t, hard[:10])
    assert near <= NEAR_PER_SITE * n
    agree = np.repeat(~mism, 3)
    assert np.max(np.abs(got[agree] - ref[agree]), initial=0) <= 1e-5
    obs = O.observables_fp64(om, L, got)
    nv = obs[10]
    assert o["n_valid"] == nv == n
    assert abs(o["energy"] - obs[0] / nv) <= 2e-6 * max(1.0, abs(obs[0] / nv))
    np.testing.assert_allclose(o["q"], obs[1:7] / nv, rtol=0, atol=2e-8)
    # sum n: per-thread FP32 sums of up to ~100 site terms, then FP64; ~1e-9 of the sum at this size
    np.testing.assert_allclose(o["nsum"], obs[7:10], rtol=5e-9, atol=1e-6 * nv ** 0.5)
    s_ref, _ = O.largest_eigen(obs[1:7] / nv)
    assert abs(o["S"] - s_ref) < 5e-8
    if not mism.any():
        assert abs(o["acceptance"] * nv - acc) < 0.5
        assert np.float32(o["ang_var"]) == np.float32(av_next)
    else:  # each differing decision moves the accepted count by one
        assert abs(o["acceptance"] * nv - acc) <= mism.sum() + 0.5
    return ref, av_next


def test_one_sweep_of_the_256_cubed_ghrl_slab_matches_the_oracle():
    surf = [("homeotropic", 1.5, 0, 0)] * 2
    em = M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=surf)
    om = O.make_model(potential="ghrl", ghrl=O.ghrl_coefficients(1.0, 0.5, 1.5), surfaces=surf)
    om.field_dir[:] = list(em.field_dir)
    pt, ns = slab_geometry()
    L = O.Lat(NX, NY, NZ, (1, 1, 0), pt, ns)
    e = M.Engine(em, [M.Replica(nx=NX, ny=NY, nz=NZ, geometry="slab", periodic=(1, 1, 0), T=T, seed=SEED)])
    ni = z_noise(NX * NY * NZ, SEED)
    e.upload(0, ni)
    plan = e.autotune(3)
    print("autotuned plan: tile configuration %d, %d planes per segment, %d work items"
          % (plan["tile_config"], plan["planes_per_segment"], plan["work_items"]))
    ni, av = compare_one_sweep(e, om, L, ni, 0.5, 1000)
    e.upload(0, ni)
    e.set_ang_var(av, 0)
    e.sweeps(20)
    ni, av = e.download(0), e.ang_var(0)
    ni, av = compare_one_sweep(e, om, L, ni, av, 2000)
    e.set_plan(2, 0)
    e.upload(0, ni)
    e.set_ang_var(av, 0)
    e.sweeps(20)
    compare_one_sweep(e, om, L, e.download(0), e.ang_var(0), 3000)
    e.close()
