"""Batched sweeps of uneven replicas: the autotuner leaves the run exactly where it was (directors, ang_var, sweep
counter, series) and picks a plan at least as fast as the one in use, and a different tile plan changes nothing in
the site updates; CUDA-graph replay of the fused sweep gives bit-for-bit the results of direct launches, across odd
sweep counts, temperature changes and a cleared series."""
import numpy as np
import pytest

from helpers import M

pytestmark = pytest.mark.gpu

SIZES = [16, 20, 24, 32, 40, 48]


def rand_dirs(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.astype(np.float32).reshape(-1)


def make():
    reps = [M.Replica(L, L, L, T=1.0 + 0.04 * i, seed=11 + i) for i, L in enumerate(SIZES)]
    e = M.Engine(M.Model("ll"), reps, M.SCHED_CHECKER2)
    for i, L in enumerate(SIZES):
        e.upload(i, rand_dirs(L ** 3, 100 + i))
    return e


def snapshot(e):
    return ([e.download(r) for r in range(len(SIZES))], [e.ang_var(r) for r in range(len(SIZES))],
            e.sweep_counter(), e.series_length())


def test_autotune_restores_the_state_and_keeps_the_physics():
    e = make()
    e.sweeps(3, measure=True)
    before = snapshot(e)
    t = e.autotune(2)
    assert t["candidates"] >= 2 and t["threads_per_cta"] in (128, 256, 512) and t["work_items"] > 0
    assert 0 <= t["tile_config"] <= 4
    assert t["ms_per_sweep"] <= t["ms_default"] * (1 + 1e-9)
    after = snapshot(e)
    for a, b in zip(before[0], after[0]):
        assert np.array_equal(a, b)
    assert before[1:] == after[1:]
    twin = make()
    twin.sweeps(3, measure=True)
    e.sweeps(5, measure=True)
    twin.sweeps(5, measure=True)
    for r in range(len(SIZES)):
        assert np.array_equal(e.download(r), twin.download(r)), r  # same site arithmetic whatever the tiling
        # the plan may change the kernel (fused or colour passes) and with it the FP32 grouping of the site terms
        np.testing.assert_allclose(e.series(r)["energy"], twin.series(r)["energy"], rtol=2e-6, atol=0)
    e.close()
    twin.close()


@pytest.mark.parametrize("cfg", ["1", "2"], ids=["fused", "pass"])
def test_graph_replay_matches_direct_launches(cfg, monkeypatch):
    monkeypatch.setenv("MCL_FUSED_CFG", cfg)
    a, b = make(), make()
    b.set_graphs(True)
    for n, meas in [(7, True), (4, False), (3, True)]:
        a.sweeps(n, measure=meas)
        b.sweeps(n, measure=meas)
    for e in (a, b):
        e.set_temperature(0.9)
        e.sweeps(2, measure=True)
        e.clear_series()
        e.sweeps(5, measure=True)
    assert a.sweep_counter() == b.sweep_counter() == 21
    assert a.series_length() == b.series_length() == 5
    for r in range(len(SIZES)):
        assert np.array_equal(a.download(r), b.download(r)), r
        sa, sb = a.series(r), b.series(r)
        assert sa.tobytes() == sb.tobytes(), r
    a.close()
    b.close()


def test_set_plan_applies_a_plan_and_keeps_the_physics():
    a, b = make(), make()
    b.set_plan(3, 8)
    p = b.plan()
    assert (p["tile_config"], p["rows_per_tile"], p["threads_per_cta"], p["planes_per_segment"]) == (3, 16, 256, 8)
    assert p["work_items"] > 0
    with pytest.raises(M.McLicsError) as ei:
        b.set_plan(99, 0)
    assert ei.value.code == 1
    b.set_graphs(True)
    for e in (a, b):
        e.sweeps(4, measure=True)
    b.set_plan(0, 0)  # back to the fused kernel mid-run: the ping-pong buffers take over from the in-place state
    for e in (a, b):
        e.sweeps(3, measure=True)
    for r in range(len(SIZES)):
        assert np.array_equal(a.download(r), b.download(r)), r
    b.set_plan(2, 0)  # and in place again after an odd number of fused sweeps (the state sits in the second buffer)
    for e in (a, b):
        e.sweeps(2, measure=True)
    for r in range(len(SIZES)):
        assert np.array_equal(a.download(r), b.download(r)), r
    a.close()
    b.close()


def test_second_buffer_exists_only_under_a_fused_plan():
    """The in-place plans hold one director buffer; a fused plan adds the second and a colour-pass plan frees it."""
    torch = pytest.importorskip("torch")
    L = 128
    e = M.Engine(M.Model("ll"), [M.Replica(L, L, L, T=1.0, seed=5)], M.SCHED_CHECKER2)
    e.upload(0, rand_dirs(L ** 3, 7))
    buffer_bytes = 12 * L ** 3  # at least the directors themselves
    assert e.plan()["tile_config"] >= 2
    free_one = torch.cuda.mem_get_info()[0]
    e.set_plan(0, 0)
    e.sweeps(1)
    free_two = torch.cuda.mem_get_info()[0]
    assert free_one - free_two >= buffer_bytes
    e.set_plan(2, 0)
    e.sweeps(1)
    assert torch.cuda.mem_get_info()[0] - free_two >= buffer_bytes
    e.close()
