"""The random initial condition (`ic random`, src/ic.cpp:38-65 in the reference, which draws gsl_ran_dir_3d from a
taus generator): here every site's director comes from Philox stream 2 keyed by the seed, computed on the device
by mcl_random_directors. The device result must equal the oracle's restatement (oracle/mc_oracle.c
mco_random_director) bit for bit, and the directors must be isotropic unit vectors."""
import numpy as np
import pytest

from helpers import M, O


def test_oracle_random_directors_are_isotropic_unit_vectors():
    n = 60000
    v = O.random_directors(11, n).astype(np.float64)
    assert np.abs(np.linalg.norm(v, axis=1) - 1).max() < 2e-7
    # uniform on the sphere: <n> = 0 (sd 1/sqrt(3n)), <n_a n_b> = delta_ab / 3 (sd ~ 0.3/sqrt(n))
    assert np.abs(v.mean(0)).max() < 5 / np.sqrt(3 * n)
    m2 = v.T @ v / n
    assert np.abs(m2 - np.eye(3) / 3).max() < 5 * 0.3 / np.sqrt(n)
    # z is uniform in [-1, 1] (Archimedes): compare the histogram with the flat one
    h, _ = np.histogram(v[:, 2], bins=20, range=(-1, 1))
    chi2 = ((h - n / 20) ** 2 / (n / 20)).sum()
    assert chi2 < 45  # 19 degrees of freedom: p ~ 1e-3
    # different seeds, different directors; the same seed, the same ones
    assert not np.array_equal(O.random_directors(12, 100), O.random_directors(11, 100))
    assert np.array_equal(O.random_directors(11, 100), v[:100].astype(np.float32))


@pytest.mark.gpu
def test_device_random_directors_equal_oracle():
    reps = [M.Replica(17, 9, 6, "bulk", (0, 0, 0)), M.Replica(8, 8, 8, "bulk", (1, 1, 1))]
    e = M.Engine(M.Model("ll"), reps)
    seeds = [12345, (1 << 40) + 7]
    for r, s in enumerate(seeds):
        e.random_directors(r, s)
    for r, (rp, s) in enumerate(zip(reps, seeds)):
        got = e.download(r).reshape(-1, 3)
        ref = O.random_directors(s, rp.nx * rp.ny * rp.nz)
        np.testing.assert_array_equal(got, ref)
    # the ghost cells follow: a sweep after the device IC equals a sweep after uploading the same field
    e2 = M.Engine(M.Model("ll"), reps)
    for r, (rp, s) in enumerate(zip(reps, seeds)):
        e2.upload(r, O.random_directors(s, rp.nx * rp.ny * rp.nz))
    e.sweeps(2)
    e2.sweeps(2)
    for r in range(2):
        np.testing.assert_array_equal(e.download(r), e2.download(r))
    e.close()
    e2.close()


@pytest.mark.gpu
def test_device_random_directors_leave_empty_sites_along_z():
    n = 11
    H = n // 2
    N = n ** 3
    pt = np.zeros(N, np.int32)
    ns = np.zeros(3 * N, np.float32)
    for q in range(N):
        i, j, k = q % n, (q // n) % n, q // (n * n)
        r = np.sqrt(np.float32((i - H) ** 2 + (j - H) ** 2 + (k - H) ** 2))
        if r < H - 1:
            pt[q] = 1
        elif r < H + 1:
            pt[q] = 2
            ns[3 * q:3 * q + 3] = np.array([i - H, j - H, k - H], np.float32) / r
    e = M.Engine(M.Model("ll", surfaces=[("homeotropic", 1.0, 0, 0)]),
                 [M.Replica(n, n, n, "sphere", (0, 0, 0))], M.SCHED_CHECKER2_SIMPLE)
    e.set_geometry(0, pt, ns)
    e.random_directors(0, 5)
    got = e.download(0).reshape(-1, 3)
    ref = O.random_directors(5, N)
    ref[pt == 0] = [0, 0, 1]
    np.testing.assert_array_equal(got, ref)
    e.close()
