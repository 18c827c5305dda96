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


def compare_replica(o, got, ni, om, L, T, seed, t, av, dims):
    """One replica of a batched sweep against the oracle's sweep of that replica alone: the same criteria."""
    nx, ny, nz = dims
    ref = ni.copy()
    acc, av_next, dec, margin = O.sweep(om, L, ref, T, av, seed, t, O.SCHED_CHECKER2, True)
    moved_gpu = np.any(got.reshape(-1, 3) != ni.reshape(-1, 3), axis=1)
    moved_ref = np.any(ref.reshape(-1, 3) != ni.reshape(-1, 3), axis=1)
    differ = np.abs(got - ref).reshape(-1, 3).max(axis=1) > 1e-5
    same_class = np.einsum("ij,ij->i", got.reshape(-1, 3), ref.reshape(-1, 3)) > 0.999  # flips change the state too
    mism = ((moved_gpu != moved_ref) & differ) | ~same_class
    hard, near = explained_mismatches(mism, margin, nx, ny, nz, L.c.periodic, TOL)
    assert not hard, hard[:10]
    agree = np.repeat(~mism, 3)
    assert np.max(np.abs(got[agree] - ref[agree]), initial=0) <= 1e-5
    obs = O.observables_fp64(om, L, got)
    nv = obs[10]
    assert abs(o["energy"] - obs[0] / nv) <= 2e-6 * max(1.0, abs(obs[0] / nv))
    np.testing.assert_allclose(o["q"], obs[1:7] / nv, rtol=0, atol=2e-8)
    return int(mism.sum()), near, nx * ny * nz


def c3_sizes(seed=11, n=64):
    """The 64 LL replicas of the batched workload: L = 2 round(exp(U(ln 16, ln 128)) / 2) from a seeded stream."""
    rng = np.random.default_rng(seed)
    return [int(2 * round(np.exp(rng.uniform(np.log(16), np.log(128))) / 2)) for _ in range(n)]


def test_one_batched_sweep_of_64_ll_replicas_matches_the_oracle():
    """The batched workload: 64 periodic LL replicas of 16^3 to 128^3 (18.1 M sites), T = 1.0 .. 1.2, each with its
    own seed, swept together in one launch per colour pass with the autotuned plan; every replica against the
    oracle's sweep of it alone."""
    sizes = c3_sizes()
    reps = [dict(L=L, T=1.0 + 0.2 * r / 63, seed=r + 1) for r, L in enumerate(sizes)]
    e = M.Engine(M.Model("ll"), [M.Replica(p["L"], p["L"], p["L"], T=p["T"], seed=p["seed"]) for p in reps])
    states = []
    for r, p in enumerate(reps):
        rng = np.random.default_rng(500 + r)
        v = rng.normal(size=(p["L"] ** 3, 3)).astype(np.float32)
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        states.append(v.reshape(-1))
        e.upload(r, states[-1])
    plan = e.autotune(3)
    print("autotuned plan: tile configuration %d, %d planes, %d work items"
          % (plan["tile_config"], plan["planes_per_segment"], plan["work_items"]))
    for r in range(len(reps)):
        e.upload(r, states[r])
    e.set_ang_var(0.4, -1)
    e.set_sweep_counter(4000)
    e.sweeps(1, measure=True)
    om = O.make_model("ll")
    total = [0, 0, 0]
    for r, p in enumerate(reps):
        L = p["L"]
        lat = O.Lat(L, L, L, (1, 1, 1))
        m, near, n = compare_replica(e.series(r)[-1], e.download(r), states[r], om, lat, np.float32(p["T"]),
                                     p["seed"], 4000, 0.4, (L, L, L))
        total = [total[0] + m, total[1] + near, total[2] + n]
    print("%d sites: %d decisions differ, %d next to the threshold" % (total[2], total[0], total[1]))
    assert total[1] <= NEAR_PER_SITE * total[2]
    e.close()


def test_one_batched_sweep_of_the_pear_field_slabs_matches_the_oracle():
    """The pear workload: 32 slabs of 256 x 256 x 64 (pear, planar degenerate anchoring W = 1, dipolar field along z
    at E = 0 .. 2, flip move, T = 0.5) swept together with the autotuned plan; three of them (E = 0, 0.97, 2) against
    the oracle's sweep of each alone."""
    n_rep, dims = 32, (256, 256, 64)
    surf = [("fg", 1.0, 0, 0)] * 2
    em = M.Model("pear", field_dir=(0, 0, 1), elecP=1.0, surfaces=surf)
    fields = [2.0 * i / 31 for i in range(n_rep)]
    e = M.Engine(em, [M.Replica(*dims, "slab", (1, 1, 0), T=0.5, elecE=fields[i], seed=5 + i) for i in range(n_rep)])
    nx, ny, nz = dims
    n = nx * ny * nz
    check = [0, 15, 31]
    states = {}
    for r in range(n_rep):
        rng = np.random.default_rng(900 + r)
        v = rng.normal(size=(n, 3)).astype(np.float32)
        v[:, 2] += 1.0
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        e.upload(r, v.reshape(-1))
        if r in check:
            states[r] = v.reshape(-1)
    plan = e.autotune(3)
    print("autotuned plan: tile configuration %d, %d planes, %d work items"
          % (plan["tile_config"], plan["planes_per_segment"], plan["work_items"]))
    for r in check:
        e.upload(r, states[r])
    e.set_ang_var(0.3, -1)
    e.set_sweep_counter(6000)
    e.sweeps(1, measure=True)
    pt = np.ones(n, np.int32)
    ns = np.zeros(3 * n, np.float32)
    plane = nx * ny
    pt[:plane] = 2
    ns[2:3 * plane:3] = -1
    pt[-plane:] = 3
    ns[3 * (n - plane) + 2::3] = 1
    lat = O.Lat(nx, ny, nz, (1, 1, 0), pt, ns)
    for r in check:
        om = O.make_model(potential="pear", field_dir=(0, 0, 1), elecP=1.0, elecE=fields[r], surfaces=surf)
        om.field_dir[:] = list(em.field_dir)
        m, near, sites = compare_replica(e.series(r)[-1], e.download(r), states[r], om, lat, np.float32(0.5), 5 + r,
                                         6000, 0.3, dims)
        print("replica %d (E = %.3f): %d decisions differ, %d next to the threshold" % (r, fields[r], m, near))
        assert near <= NEAR_PER_SITE * sites
    e.close()
