"""mcl_sweeps_io (temperatures up, measured sweeps, records down, one synchronisation) against the three-call
sequence it replaces (mcl_set_temperature per replica, mcl_sweeps, mcl_read_series; the measurement loop of
src/evolve_thermal.cu:78-106): identical records and directors, on one and on several replicas, the plain and the
learned proposal, with and without CUDA graphs; argument errors leave the engine usable."""
import numpy as np
import pytest

from helpers import M
from oracle import learned as L

pytestmark = pytest.mark.gpu


def rand_dirs(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.astype(np.float32).reshape(-1)


def make(model, sizes, geometry="bulk"):
    reps = [M.Replica(n, n, n, T=1.0, seed=5 + i, geometry=geometry) for i, n in enumerate(sizes)]
    e = M.Engine(model, reps, M.SCHED_CHECKER2)
    for i, n in enumerate(sizes):
        e.upload(i, rand_dirs(n ** 3, 40 + i))
    return e


def three_calls(e, n, T):
    first = e.series_length()
    for r, t in enumerate(T):
        e.set_temperature(float(t), r)
    e.sweeps(n, measure=True)
    recs = [e.series(r, first, n) for r in range(e.n)]
    return np.stack(recs, axis=1).reshape(-1)  # [sweep][replica]


@pytest.mark.parametrize("graphs", [False, True], ids=["direct", "graph"])
@pytest.mark.parametrize("sizes", [[32], [16, 24, 20]], ids=["one", "three"])
def test_sweeps_io_matches_the_three_calls(sizes, graphs):
    a, b = make(M.Model("ll"), sizes), make(M.Model("ll"), sizes)
    for e in (a, b):
        e.set_graphs(graphs)
    temps = [np.linspace(0.6, 1.2, len(sizes)).astype(np.float32), np.full(len(sizes), 0.9, np.float32)]
    for step, n in enumerate([1, 3, 2, 1]):
        T = temps[step % 2]
        got = a.sweeps_io(n, T)
        want = three_calls(b, n, T)
        assert got.shape == want.shape == (n * len(sizes),)
        assert got.tobytes() == want.tobytes(), (step, n)
    out = np.zeros(2 * len(sizes), M.OBS_DTYPE)
    got = a.sweeps_io(2, None, out)  # None keeps the temperatures
    assert got is out
    want = three_calls(b, 2, temps[1])
    assert out.tobytes() == want.tobytes()
    for r in range(len(sizes)):
        assert np.array_equal(a.download(r), b.download(r))
    assert a.series_length() == b.series_length()
    a.close()
    b.close()


def test_sweeps_io_with_the_learned_proposal():
    sizes = [24]
    model = M.Model("ll")
    a, b = make(model, sizes), make(model, sizes)
    params = L.init_params(3).astype(np.float32)
    for e in (a, b):
        e.set_proposal(params)
    T = np.array([0.8], np.float32)
    got = a.sweeps_io(3, T)
    want = three_calls(b, 3, T)
    assert got.tobytes() == want.tobytes()
    assert np.array_equal(a.download(0), b.download(0))
    a.close()
    b.close()


def test_sweeps_io_refuses_bad_arguments_and_stays_usable():
    e = make(M.Model("ll"), [16, 16])
    for bad in ([-1.0, 1.0], [1.0, float("nan")], [float("inf"), 1.0]):
        with pytest.raises(M.McLicsError):
            e.sweeps_io(1, np.array(bad, np.float32))
    with pytest.raises(ValueError):
        e.sweeps_io(1, np.array([1.0], np.float32))
    with pytest.raises(M.McLicsError):
        M.check(M.lib().mcl_sweeps_io(e._h, 0, None, np.zeros(2, M.OBS_DTYPE).ctypes.data))
    assert e.series_length() == 0
    recs = e.sweeps_io(2, np.array([1.0, 1.1], np.float32))
    assert recs.size == 4 and np.all(np.isfinite(recs["energy"])) and np.all(recs["n_valid"] == 16 ** 3)
    assert recs["sweep"][0] == recs["sweep"][1] and recs["sweep"][2] == recs["sweep"][3] > recs["sweep"][0]
    e.close()


@pytest.mark.parametrize("io", [False, True], ids=["sweeps", "sweeps_io"])
def test_adaptation_switch_reaches_captured_graphs(io):
    """ang_var adaptation is an argument of the captured finalisation: switching it off after a graph was captured
    must stop the adaptation in the graph replays too (mcl_sweeps and mcl_sweeps_io's one-step graph)."""
    e = make(M.Model("ll"), [16])
    e.set_graphs(True)
    T = np.array([1.0], np.float32)

    def run(k):
        if io:
            for _ in range(k):
                e.sweeps_io(1, T)
        else:
            e.sweeps(k, measure=True)

    run(4)  # captures with adaptation on
    a0 = e.ang_var(0)
    run(4)
    assert e.ang_var(0) != a0  # adapting
    e.set_adaptation(False)
    a1 = e.ang_var(0)
    run(6)
    assert e.ang_var(0) == a1
    e.set_adaptation(True)
    run(4)
    assert e.ang_var(0) != a1
    e.close()


def test_reserved_series_keeps_the_records():
    """mcl_reserve_series sizes the series once; the records and directors of the sweeps that follow are those of an
    engine that grows its series as it goes (graphs on, so a reallocation also means a new capture)."""
    a, b = make(M.Model("ll"), [16, 20]), make(M.Model("ll"), [16, 20])
    for e in (a, b):
        e.set_graphs(True)
    a.reserve_series(500)
    a.reserve_series(10)  # smaller than the capacity: nothing changes
    T = np.array([0.9, 1.1], np.float32)
    for _ in range(3):
        a.sweeps(70, measure=True)
        b.sweeps(70, measure=True)
        ra, rb = a.sweeps_io(1, T), b.sweeps_io(1, T)
        assert ra.tobytes() == rb.tobytes()
    assert a.series_length() == b.series_length() == 213
    for r in range(2):
        assert a.series(r).tobytes() == b.series(r).tobytes()
        assert np.array_equal(a.download(r), b.download(r))
    with pytest.raises(M.McLicsError):
        a.reserve_series(-1)
    a.close()
    b.close()
