"""Device-side extra order parameters (P, dtheta, divn, radial Sr/Pr; mcl_measure_extras) against the CPU
restatement of src/parameter_order.cpp:129-245 (oracle/extras.py) on random and structured lattices: periodic and
free bulk, a slab, and a sphere with empty sites."""
import numpy as np
import pytest

from helpers import M
from oracle import extras as X

pytestmark = pytest.mark.gpu


def dirs(n, seed, bias):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v += np.asarray(bias)
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.astype(np.float32)


def hedgehog(nx, ny, nz):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    r = np.stack([i - nx // 2, j - ny // 2, k - nz // 2], -1).astype(np.float64)
    r = r.transpose(2, 1, 0, 3).reshape(-1, 3)
    nrm = np.linalg.norm(r, axis=1)
    r[nrm == 0] = (0, 0, 1)
    return (r / np.linalg.norm(r, axis=1)[:, None]).astype(np.float32)


CASES = [
    ("pear_bulk_periodic", "bulk", (1, 1, 1), (10, 8, 6), "random"),
    ("pear_bulk_free", "bulk", (0, 0, 0), (9, 7, 5), "random"),
    ("pear_slab", "slab", (1, 1, 0), (8, 8, 7), "random"),
    ("pear_sphere_hedgehog", "sphere", (0, 0, 0), (12, 12, 12), "hedgehog"),
]


@pytest.mark.parametrize("name,geo,per,shape,kind", CASES, ids=[c[0] for c in CASES])
def test_extras_match_reference_formulas(name, geo, per, shape, kind):
    nx, ny, nz = shape
    n = nx * ny * nz
    surfaces = [("fg", 1.0, 0, 0)] * (2 if geo == "slab" else 1 if geo == "sphere" else 0)
    e = M.Engine(M.Model("pear", surfaces=surfaces), [M.Replica(nx, ny, nz, geo, per, T=0.5, seed=3)])
    ni = hedgehog(nx, ny, nz) if kind == "hedgehog" else dirs(n, 7, (0.3, -0.2, 1.0))
    e.upload(0, ni.reshape(-1))
    e.sweeps(2)
    cur = e.download(0).reshape(-1, 3)
    o = e.measure(0)
    got = e.measure_extras(0, o["director"])
    if geo == "sphere":
        # point types of the sphere geometry (src/geometry_sphere.cpp:32-58), as the engine builds them
        i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        H = np.float32(nz // 2)
        r = np.sqrt(((i - np.float32(nx // 2)) ** 2 + (j - np.float32(ny // 2)) ** 2 + (k - H) ** 2).astype(np.float32))
        pt = np.where(r < H - 1, 1, np.where(r < H + 1, 2, 0)).transpose(2, 1, 0).reshape(-1)
    else:
        pt = np.ones(n, int)
    periodic = [bool(p) for p in per]
    if geo == "slab":
        periodic[2] = False
    if geo == "sphere":
        periodic = [False] * 3
    ref = X.extras(cur, pt, shape, periodic, np.asarray(o["director"], np.float32))
    for key in ref:
        assert abs(got[key] - ref[key]) <= 2e-6 + 2e-6 * abs(ref[key]), (key, got[key], ref[key])
    if kind == "hedgehog":
        assert got["Sr_sph"] > 0.5  # radial; the polar sign is scrambled by the flip moves
    e.close()


@pytest.mark.parametrize("geo,per,shape", [("bulk", (1, 1, 1), (6, 4, 4)), ("slab", (0, 1, 0), (5, 6, 5)),
                                           ("sphere", (0, 0, 0), (8, 8, 8))])
def test_local_order_matches_reference_formula(geo, per, shape):
    nx, ny, nz = shape
    n = nx * ny * nz
    surfaces = [("homeotropic", 1.0, 0, 0)] * (2 if geo == "slab" else 1 if geo == "sphere" else 0)
    e = M.Engine(M.Model("ll", surfaces=surfaces), [M.Replica(nx, ny, nz, geo, per, T=0.8, seed=5)])
    e.upload(0, dirs(n, 11, (0.2, 0.1, 0.8)).reshape(-1))
    e.sweeps(3)
    cur = e.download(0).reshape(-1, 3)
    S = e.local_order(0)
    periodic = [bool(p) for p in per]
    if geo == "sphere":
        i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        H = np.float32(nz // 2)
        r = np.sqrt(((i - np.float32(nx // 2)) ** 2 + (j - np.float32(ny // 2)) ** 2 + (k - H) ** 2).astype(np.float32))
        pt = np.where(r < H - 1, 1, np.where(r < H + 1, 2, 0)).transpose(2, 1, 0).reshape(-1)
    else:
        pt = np.ones(n, int)
    for q in range(n):
        if not pt[q]:
            assert np.isnan(S[q])
            continue
        i, j, k = q % nx, (q // nx) % ny, q // (nx * ny)
        ref = X.local_S(cur, pt, shape, periodic, i, j, k)
        assert abs(S[q] - ref) <= 1e-6 + 1e-6 * abs(ref), (q, S[q], ref)
    e.close()
