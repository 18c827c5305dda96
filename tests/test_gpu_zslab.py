"""The z-slab decomposition on one GPU: the ranks of a decomposition run as slabs of one process (LocalGroup:
device copies as the exchange, a sum as the all-reduce) and must reproduce one engine sweeping the whole lattice
bit for bit — the owned planes of every slab equal the whole lattice's planes, and every slab's series equals the
whole engine's (acceptance and ang_var exactly; E, Q, S up to the order of the FP64 sums). Cases: periodic bulk
with even and uneven splits, a slab with anchoring on the planes of the end ranks, a flip + field model, and one
periodic rank exchanging with itself."""
import numpy as np
import pytest

from helpers import M

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from mclics_b200 import zslab  # noqa: E402


def rand_dirs(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.astype(np.float32).reshape(-1)


MODELS = {
    "ll": lambda: M.Model("ll"),
    "ghrl_slab": lambda: M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=[("homeotropic", 1.5, 0, 0)] * 2),
    "pear_field": lambda: M.Model("pear", A=1.5, B1=0.09, C=0.3, field_dir=(0.3, 0, 1), elecP=0.7, elecA=0.1,
                                  surfaces=[("fg", 1.0, 0, 0), ("rp", 0.5, 40, 10)]),
}

CASES = [
    # (model, nx, ny, nz, geometry, periodic xy, periodic z, world)
    ("ll", 40, 20, 30, "bulk", (1, 1), True, 3),
    ("ll", 40, 20, 30, "bulk", (1, 1), True, 4),      # 8, 8, 7, 7 planes
    ("ll", 36, 18, 30, "bulk", (0, 1), False, 2),     # free x and z
    ("ghrl_slab", 36, 18, 21, "slab", (1, 1), False, 3),
    ("pear_field", 34, 14, 16, "slab", (1, 1), False, 2),
    ("ll", 32, 16, 12, "bulk", (1, 1), True, 1),      # one rank: its halos are its own boundary planes
]


def whole(model, nx, ny, nz, geo, pxy, pz, ni, sweeps):
    e = M.Engine(model, [M.Replica(nx, ny, nz, geo, (pxy[0], pxy[1], 1 if pz else 0), T=0.9, seed=99)])
    e.upload(0, ni)
    e.set_sweep_counter(17)
    e.sweeps(sweeps, measure=True)
    out, ser = e.download(0), e.series(0)
    e.close()
    return out, ser


@pytest.mark.parametrize("case", CASES, ids=["%s-%dx%dx%d-%s-z%s-w%d" % (c[0], c[1], c[2], c[3], c[4], int(c[6]), c[7])
                                             for c in CASES])
def test_slabs_reproduce_the_whole_lattice(case):
    name, nx, ny, nz, geo, pxy, pz, world = case
    model = MODELS[name]()
    ni = rand_dirs(nx * ny * nz, 5)
    K = 4
    ref, ref_ser = whole(model, nx, ny, nz, geo, pxy, pz, ni, K)
    stream = torch.cuda.Stream()
    slabs = [zslab.ZSlab(model, nx, ny, nz, r, world, None, geometry=geo, periodic_xy=pxy, periodic_z=pz, T=0.9,
                         seed=99, stream=stream) for r in range(world)]
    for s in slabs:
        s.upload_global(ni)
        s.set_sweep_counter(17)
    group = zslab.LocalGroup(slabs)
    group.sweeps(2, measure=True)
    group.sweeps(K - 2, measure=True)
    got = np.concatenate([s.download_owned() for s in slabs])
    np.testing.assert_array_equal(got, ref)
    for s in slabs:
        ser = s.series()
        assert len(ser) == K
        np.testing.assert_array_equal(ser["acceptance"], ref_ser["acceptance"])
        np.testing.assert_array_equal(ser["ang_var"], ref_ser["ang_var"])
        np.testing.assert_array_equal(ser["sweep"], ref_ser["sweep"])
        # a slab's work items end at its own planes, so the per-thread FP32 sums group the site terms differently
        # from the whole lattice's (FP64 beyond the thread): agreement to FP32 rounding of those small groups
        np.testing.assert_allclose(ser["energy"], ref_ser["energy"], rtol=1e-7, atol=0)
        np.testing.assert_allclose(ser["q"], ref_ser["q"], rtol=0, atol=1e-8)
        np.testing.assert_allclose(ser["S"], ref_ser["S"], rtol=0, atol=1e-8)
        np.testing.assert_allclose(ser["nsum"], ref_ser["nsum"], rtol=0, atol=1e-6 * (nx * ny * nz) ** 0.5)
        assert np.all(ser["n_valid"] == nx * ny * nz)
    for s in slabs:
        s.eng.close()


def test_slab_engine_refuses_whole_lattice_calls():
    s = zslab.ZSlab(M.Model("ll"), 32, 16, 12, 0, 2, None, periodic_z=True, seed=3)
    for call in (lambda: s.eng.sweeps(1), lambda: s.eng.measure(0), lambda: s.eng.autotune(1),
                 lambda: s.eng.set_plan(1, 0), lambda: s.eng.sweeps_io(1, np.array([1.0], np.float32))):
        with pytest.raises(M.McLicsError) as ei:
            call()
        assert ei.value.code == 4
    s.eng.close()
