"""The tiled sweeps on TMA-streamed planes — the fused kernel (both colours per pass over HBM, ghost cells,
ping-pong buffers) and the in-place colour passes — against the untiled two-colour kernel: same Philox draws, same
physics code, so they must agree site by site on every geometry the tiling has to get right (ragged last tiles,
several z segments, free and periodic axes, tiny lattices, batches of replicas of different sizes). The colour
passes must reproduce the fused kernel bit for bit in every tile configuration. Also the bounded TMA wait: a
withheld copy makes the wait run out, the error is reported at the next synchronising call and the engine keeps
working."""
import numpy as np
import pytest

# tile configurations (MCL_FUSED_CFG): "0", "1" = fused kernel (64 x 14, 64 x 28 tiles), "2"-"4" = colour passes
# (64 x 16 at 3 or 2 CTAs per SM, 32 x 16)
KERNELS = {"fused14": "0", "fused28": "1", "pass": "2", "pass32": "4"}
PASS_CFGS = ["2", "3", "4"]


@pytest.fixture
def kernel_cfg(monkeypatch, request):
    cfg = request.param
    if cfg is None:
        monkeypatch.delenv("MCL_FUSED_CFG", raising=False)
    else:
        monkeypatch.setenv("MCL_FUSED_CFG", cfg)
    return cfg

from helpers import M


def rand_dirs(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3)).astype(np.float32)
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.reshape(-1).astype(np.float32)


MODELS = {
    "ll": lambda: M.Model("ll"),
    "ghrl_slab": lambda: M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=[("homeotropic", 1.5, 0, 0)] * 2),
    "ghrl_chiral_rp": lambda: M.Model("ghrl", k=(1.48, 1, 2.28, 12.0),
                                      surfaces=[("rp_ghrl", 1.0, 90, 30), ("fg_ghrl", 0.8, 0, 0)]),
    "pear_field": lambda: M.Model("pear", A=1.5, B1=0.09, C=0.3, field_dir=(0.3, 0, 1), elecP=0.7, elecA=0.1,
                                  surfaces=[("fg", 1.0, 0, 0), ("rp", 0.5, 40, 10)]),
}

SHAPES = [
    # (nx, ny, nz, geometry, periodic)
    (64, 16, 40, "bulk", (1, 1, 1)),
    (72, 22, 70, "bulk", (1, 1, 1)),       # ragged x and y tiles, several z segments
    (30, 18, 26, "bulk", (0, 0, 0)),       # free everywhere, odd-free sizes
    (2, 2, 2, "bulk", (1, 1, 1)),          # smallest periodic lattice: ghosts of ghosts
    (6, 4, 4, "bulk", (1, 0, 1)),          # periodic nx % 4 == 2: the right ring site shares a pair of cells
    (66, 12, 10, "bulk", (1, 1, 1)),       # ... also in a second x tile
    (68, 20, 33, "slab", (1, 1, 0)),
    (16, 16, 1, "slab", (1, 1, 0)),        # single plane (surface 1 only)
    (130, 34, 12, "slab", (0, 1, 0)),
    (29, 10, 9, "bulk", (0, 0, 0)),        # odd nx along a free x: a pair task whose first site is beyond the edge
]


def run(model, reps, schedule, sweeps, measure, seeds):
    e = M.Engine(model, reps, schedule)
    for r, rp in enumerate(reps):
        e.upload(r, rand_dirs(rp.nx * rp.ny * rp.nz, seeds[r]))
    e.set_sweep_counter(17)
    e.sweeps(sweeps, measure=measure)
    out = [e.download(r) for r in range(len(reps))]
    ser = [e.series(r) for r in range(len(reps))] if measure else None
    av = [e.ang_var(r) for r in range(len(reps))]
    e.close()
    return out, ser, av


SHAPE_IDS = ["%dx%dx%d-%s-%s" % (s[0], s[1], s[2], s[3], "".join(map(str, s[4]))) for s in SHAPES]


def model_for(model, geo):
    if geo == "bulk" and model in ("ghrl_slab", "ghrl_chiral_rp", "pear_field"):
        m = MODELS[model]()
        m.n_surfaces = 0
    else:
        m = MODELS[model]()
    if geo == "slab" and m.n_surfaces < 2:
        m = M.Model("ll", surfaces=[("homeotropic", 1.0, 0, 0), ("fg", 0.5, 0, 0)])
    return m


@pytest.mark.gpu
@pytest.mark.parametrize("kernel_cfg", list(KERNELS.values()), ids=list(KERNELS), indirect=True)
@pytest.mark.parametrize("model", sorted(MODELS))
@pytest.mark.parametrize("shape", SHAPES, ids=SHAPE_IDS)
def test_fused_equals_untiled(model, shape, kernel_cfg):
    nx, ny, nz, geo, per = shape
    m = model_for(model, geo)
    reps = [M.Replica(nx, ny, nz, geo, per, T=0.9, seed=99)]
    a, sa, ava = run(m, reps, M.SCHED_CHECKER2, 4, True, [5])
    b, sb, avb = run(m, reps, M.SCHED_CHECKER2_SIMPLE, 4, True, [5])
    diff = np.abs(a[0] - b[0])
    assert diff.max() <= 2e-6, "max director difference %g" % diff.max()
    assert ava == avb
    np.testing.assert_allclose(sa[0]["energy"], sb[0]["energy"], rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(sa[0]["q"], sb[0]["q"], rtol=0, atol=2e-7)
    np.testing.assert_array_equal(sa[0]["acceptance"], sb[0]["acceptance"])


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", PASS_CFGS)
@pytest.mark.parametrize("model", sorted(MODELS))
@pytest.mark.parametrize("shape", SHAPES, ids=SHAPE_IDS)
def test_colour_passes_equal_fused_bitwise(model, shape, cfg, monkeypatch):
    nx, ny, nz, geo, per = shape
    m = model_for(model, geo)
    reps = [M.Replica(nx, ny, nz, geo, per, T=0.9, seed=99)]
    monkeypatch.setenv("MCL_FUSED_CFG", "1")
    a, sa, ava = run(m, reps, M.SCHED_CHECKER2, 5, True, [5])
    monkeypatch.setenv("MCL_FUSED_CFG", cfg)
    b, sb, avb = run(m, reps, M.SCHED_CHECKER2, 5, True, [5])
    np.testing.assert_array_equal(a[0], b[0])
    assert ava == avb
    np.testing.assert_allclose(sa[0]["energy"], sb[0]["energy"], rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(sa[0]["q"], sb[0]["q"], rtol=0, atol=2e-7)
    np.testing.assert_allclose(sa[0]["nsum"], sb[0]["nsum"], rtol=1e-6, atol=1e-4)
    np.testing.assert_array_equal(sa[0]["acceptance"], sb[0]["acceptance"])


@pytest.mark.gpu
@pytest.mark.parametrize("plan", [(2, 2), (3, 2), (4, 2), (4, 3)], ids=["2,2", "3,2", "4,2", "4,3"])
@pytest.mark.parametrize("model", ["ll", "ghrl_slab", "pear_field"])
@pytest.mark.parametrize("shape", [SHAPES[0], SHAPES[2], SHAPES[6]], ids=[SHAPE_IDS[0], SHAPE_IDS[2], SHAPE_IDS[6]])
def test_short_segments_equal_fused_bitwise(plan, model, shape, monkeypatch):
    """Colour passes with segments of 2 and 3 planes (the autotuner's candidates for lattices that give fewer work
    items than SMs): the same directors, acceptance and ang_var as the fused kernel."""
    nx, ny, nz, geo, per = shape
    m = model_for(model, geo)
    reps = [M.Replica(nx, ny, nz, geo, per, T=0.9, seed=99)]
    monkeypatch.setenv("MCL_FUSED_CFG", "1")
    a, sa, ava = run(m, reps, M.SCHED_CHECKER2, 5, True, [5])
    monkeypatch.delenv("MCL_FUSED_CFG", raising=False)
    e = M.Engine(m, reps, M.SCHED_CHECKER2)
    e.upload(0, rand_dirs(nx * ny * nz, 5))
    e.set_plan(*plan)
    assert e.plan()["planes_per_segment"] == min(plan[1], nz)
    e.set_sweep_counter(17)
    e.sweeps(5, measure=True)
    b, sb, avb = e.download(0), e.series(0), e.ang_var(0)
    e.close()
    np.testing.assert_array_equal(a[0], b)
    assert ava[0] == avb
    np.testing.assert_array_equal(sa[0]["acceptance"], sb["acceptance"])
    np.testing.assert_allclose(sa[0]["energy"], sb["energy"], rtol=2e-6, atol=2e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel_cfg", list(KERNELS.values()), ids=list(KERNELS), indirect=True)
def test_fused_batch_of_uneven_replicas(kernel_cfg):
    m = M.Model("ll")
    sizes = [(16, 16, 16), (24, 24, 24), (40, 18, 30), (8, 8, 8), (64, 32, 20)]
    reps = [M.Replica(*s, T=1.0 + 0.05 * i, seed=100 + i) for i, s in enumerate(sizes)]
    a, sa, ava = run(m, reps, M.SCHED_CHECKER2, 3, True, list(range(len(sizes))))
    for i, s in enumerate(sizes):
        b, sb, avb = run(m, [reps[i]], M.SCHED_CHECKER2_SIMPLE, 3, True, [i])
        assert np.abs(a[i] - b[0]).max() <= 2e-6
        np.testing.assert_allclose(sa[i]["energy"], sb[0]["energy"], rtol=2e-6)
        assert ava[i] == avb[0]


@pytest.mark.gpu
@pytest.mark.parametrize("kernel_cfg", list(KERNELS.values()), ids=list(KERNELS), indirect=True)
def test_ghosts_and_buffers_survive_alternating_paths(kernel_cfg):
    """Fused sweeps, then untiled ones (decision recording forces them), then fused again: the ghost cells and the
    ping-pong buffers stay consistent with an engine that used the untiled path throughout."""
    m = M.Model("ghrl", k=(1.0, 0.5, 1.5))
    rp = M.Replica(40, 20, 24, "bulk", (1, 1, 1), T=0.8, seed=3)
    e1 = M.Engine(m, [rp], M.SCHED_CHECKER2)
    e2 = M.Engine(m, [rp], M.SCHED_CHECKER2_SIMPLE)
    x = rand_dirs(40 * 20 * 24, 9)
    for e in (e1, e2):
        e.upload(0, x)
    e1.sweeps(2)
    e1.record_decisions(True)
    e1.sweeps(2)
    e1.record_decisions(False)
    e1.sweeps(3)
    e2.sweeps(7)
    assert np.abs(e1.download(0) - e2.download(0)).max() <= 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("kernel_cfg", list(KERNELS.values()), ids=list(KERNELS), indirect=True)
def test_tma_wait_timeout_reports_and_recovers(kernel_cfg):
    m = M.Model("ll")
    rp = M.Replica(64, 32, 32, "bulk", (1, 1, 1), T=1.0, seed=1)
    e = M.Engine(m, [rp], M.SCHED_CHECKER2)
    x = rand_dirs(64 * 32 * 32, 1)
    e.upload(0, x)
    e.debug_wait_limit(100_000_000, withhold_first_load=True)  # 0.1 s
    e.sweeps(1)
    with pytest.raises(M.McLicsError) as ei:
        e.synchronize()
    assert ei.value.code == 2 and "did not complete" in str(ei.value)
    e.debug_wait_limit(2_000_000_000, withhold_first_load=False)
    e.upload(0, x)
    e.sweeps(3, measure=True)
    e.synchronize()
    s = e.series(0)
    assert np.all(np.isfinite(s["energy"])) and s["energy"][-1] < 0
