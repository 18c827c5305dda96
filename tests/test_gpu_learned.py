"""The learned MH proposal on the GPU against the FP64 oracle (oracle/learned.py): the tensor-core MLP forward pass,
the features of extracted training samples, the training gradient, and that training lowers the loss. Then the
property that makes the proposal usable at all: learned sweeps leave the Boltzmann distribution unchanged, so
<E> and <S> agree with the plain sweep's within their statistical errors, for trained and for untrained
weights."""
import numpy as np
import pytest

from helpers import M
from oracle import learned as L

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rand_dirs(n, seed, bias=0.0):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v[:, 2] += bias
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.astype(np.float32).reshape(-1)


def perturbed_params(seed):
    rng = np.random.default_rng(seed)
    p = L.init_params(3)
    return (p + 0.3 * rng.normal(size=p.size) * np.abs(p).mean()).astype(np.float32)


def engine_ll(L_, T, seed, n_rep=1, sweeps=0):
    reps = [M.Replica(L_, L_, L_, T=T, seed=seed + r) for r in range(n_rep)]
    e = M.Engine(M.Model("ll"), reps, M.SCHED_CHECKER2)
    for r in range(n_rep):
        e.upload(r, rand_dirs(L_ ** 3, seed + 100 * r, bias=1.5))
    if sweeps:
        e.sweeps(sweeps)
    return e


def extract(e, r, n, seed):
    feat = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    dirs = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    e.extract_samples(r, n, seed, feat.data_ptr(), dirs.data_ptr())
    return feat, dirs


def test_mlp_forward_matches_oracle():
    rng = np.random.default_rng(2)
    n = 5000
    x = np.zeros((n, 8), np.float32)
    x[:, :6] = rng.uniform(-0.5, 1.0, (n, 6))
    x[:, 6] = rng.uniform(0.2, 1.3, n)
    x[:, 7] = 1
    p = perturbed_params(4)
    feat = torch.from_numpy(x).cuda()
    out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    M.mlp_forward(p, feat.data_ptr(), n, out.data_ptr())
    got = out.cpu().numpy().astype(np.float64)
    ref, _ = L.forward(p.astype(np.float64), x[:, :7].astype(np.float64))
    # same BF16 operands; FP32 sums in another order can move a hidden activation across a BF16 rounding step
    err = np.abs(got - ref)
    assert err.max() < 3e-2, err.max()
    assert err.mean() < 2e-3, err.mean()


def test_tcgen05_forward_matches_mma_sync_and_oracle():
    rng = np.random.default_rng(8)
    n = 5000  # 19 full chunks of 256 rows and a ragged one
    x = np.zeros((n, 8), np.float32)
    x[:, :6] = rng.uniform(-0.5, 1.0, (n, 6))
    x[:, 6] = rng.uniform(0.2, 1.3, n)
    x[:, 7] = 1
    p = perturbed_params(6)
    feat = torch.from_numpy(x).cuda()
    out_tc = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda")
    out_mma = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    M.mlp_forward(p, feat.data_ptr(), n, out_tc.data_ptr(), tcgen05=True)
    M.mlp_forward(p, feat.data_ptr(), n, out_mma.data_ptr())
    a, b = out_tc.cpu().numpy().astype(np.float64), out_mma.cpu().numpy().astype(np.float64)
    assert np.isfinite(a).all()
    ref, _ = L.forward(p.astype(np.float64), x[:, :7].astype(np.float64))
    # same BF16 operands and FP32 accumulation, sums in another order
    assert np.abs(a - b).max() < 3e-2 and np.abs(a - b).mean() < 1e-3, (np.abs(a - b).max(), np.abs(a - b).mean())
    assert np.abs(a - ref).max() < 3e-2 and np.abs(a - ref).mean() < 2e-3


def test_extracted_features_match_oracle():
    nx = 10
    e = engine_ll(nx, 0.8, 5)
    ni = e.download(0).reshape(-1, 3)
    feat, dirs = extract(e, 0, 3000, 17)
    f = feat.cpu().numpy()
    d = dirs.cpu().numpy()
    assert np.all(f[:, 7] == 1)
    index = {tuple(v): i for i, v in enumerate(ni)}
    sites = np.array([index[tuple(v)] for v in d])
    assert len(np.unique(sites)) > 900  # the draws cover the lattice
    x, y, z = sites % nx, (sites // nx) % nx, sites // (nx * nx)
    nbr = []
    for dx, dy, dz in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
        nbr.append(ni[((x + dx) % nx) + nx * (((y + dy) % nx) + nx * ((z + dz) % nx))])
    ref = L.features(np.stack(nbr, 1), np.ones((len(sites), 6)), 0.8)
    np.testing.assert_allclose(f[:, :7], ref, rtol=0, atol=2e-6)
    e.close()


def test_gradient_matches_oracle():
    e = engine_ll(16, 0.6, 7, sweeps=30)
    n = 1024
    feat, dirs = extract(e, 0, n, 3)
    p = perturbed_params(5)
    # the axis gradient scales as 1 / |o[0:3]|; a clear axis bias keeps every sample well conditioned, so the
    # one-ulp BF16 differences of hidden activations between the FP32 and FP64 sums stay small in the gradient
    p[-2] += 3.0
    t = M.Trainer(p, n)
    loss, g = t.gradient(feat.data_ptr(), dirs.data_ptr(), n)
    x = feat.cpu().numpy()[:, :7].astype(np.float64)
    d = dirs.cpu().numpy().astype(np.float64)
    o, _ = L.forward(p.astype(np.float64), x)
    assert np.linalg.norm(o[:, :3], axis=1).min() > 1.0
    ref_loss, ref_g = L.loss_and_grad(p.astype(np.float64), x, d)
    assert abs(loss - ref_loss) < 1e-4 * max(1.0, abs(ref_loss)), (loss, ref_loss)
    scale = np.abs(ref_g).max()
    assert np.abs(g - ref_g).max() < 5e-3 * scale, (np.abs(g - ref_g).max(), scale)
    assert np.linalg.norm(g - ref_g) < 1e-2 * np.linalg.norm(ref_g)
    t.close()
    e.close()


def train_on(e, n_rep, steps, seed=3, batch=4096, lr=3e-3, snapshots=8, per=4096):
    """Samples from `snapshots` states of every replica (5 sweeps apart), then `steps` Adam steps."""
    n = snapshots * n_rep * per
    feat = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    dirs = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    k = 0
    for s in range(snapshots):
        e.sweeps(5)
        for r in range(n_rep):
            e.extract_samples(r, per, seed * 1000 + s * 17 + r, feat[k:].data_ptr(), dirs[k:].data_ptr())
            k += per
    g = torch.Generator(device="cpu").manual_seed(seed)
    t = M.Trainer(L.init_params(seed).astype(np.float32), batch)
    losses = []
    for i in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g).cuda()
        fb, db = feat[idx].contiguous(), dirs[idx].contiguous()
        losses.append(t.step(fb.data_ptr(), db.data_ptr(), batch, lr))
    p = t.params()
    t.close()
    return p, losses


def test_training_lowers_the_loss():
    e = engine_ll(16, 0.5, 11, n_rep=2, sweeps=200)
    p, losses = train_on(e, 2, 300)
    first, last = np.mean(losses[:10]), np.mean(losses[-20:])
    # 0 is the loss of the uniform proposal; the local conditional at T = 0.5 is far narrower
    assert last < first - 0.5 and last < -0.5, (first, last)
    # and the trained proposal is accepted far more often than the untrained one
    e.set_proposal(p)
    e.sweeps(20, measure=True)
    acc_trained = e.series(0)["acceptance"][-10:].mean()
    e.set_proposal(L.init_params(3).astype(np.float32))
    e.clear_series()
    e.sweeps(20, measure=True)
    acc_init = e.series(0)["acceptance"][-10:].mean()
    assert acc_trained > 0.4 and acc_trained > acc_init + 0.1, (acc_trained, acc_init)
    e.close()


def replica_means(e, n_rep, therm, meas):
    e.sweeps(therm)
    e.clear_series()
    e.sweeps(meas, measure=True)
    E = np.array([e.series(r)["energy"].mean() for r in range(n_rep)])
    S = np.array([e.series(r)["S"].mean() for r in range(n_rep)])
    return E, S


@pytest.mark.parametrize("trained", [False, True])
def test_learned_sweep_keeps_the_equilibrium(trained):
    T, n_rep, nx = 0.7, 8, 12
    plain = engine_ll(nx, T, 21, n_rep=n_rep)
    E0, S0 = replica_means(plain, n_rep, 600, 3000)
    learned = engine_ll(nx, T, 61, n_rep=n_rep)
    if trained:
        learned.sweeps(200)
        p, _ = train_on(learned, n_rep, 200, snapshots=4, per=2048)
    else:
        p = perturbed_params(9)
    learned.set_proposal(p)
    E1, S1 = replica_means(learned, n_rep, 600, 3000)
    for a, b in [(E0, E1), (S0, S1)]:
        se = np.sqrt(a.var(ddof=1) / n_rep + b.var(ddof=1) / n_rep)
        assert abs(a.mean() - b.mean()) < 4 * se + 1e-4, (a.mean(), b.mean(), se)
    plain.close()
    learned.close()


def test_learned_and_mixed_sweeps_keep_the_equilibrium_near_the_transition():
    """LL at T = 1.12, just below the nematic-isotropic transition (T_NI = 1.1232), where the order fluctuates
    slowly and a bias of the proposal would show first: 32 independent 20^3 replicas per arm, the network trained
    on this lattice's own states; <E> and <S> of the learned arm and of the mixture (one learned sweep after every
    plain one) against the plain arm's, errors from the spread between replicas (independent chains: no
    autocorrelation estimate enters), within 4 combined standard errors."""
    T, n_rep, nx = 1.12, 32, 20
    plain = engine_ll(nx, T, 201, n_rep=n_rep)
    E0, S0 = replica_means(plain, n_rep, 3000, 8000)
    tr = engine_ll(nx, T, 401, n_rep=4, sweeps=1000)
    p, _ = train_on(tr, 4, 300, snapshots=4, per=4096)
    tr.close()
    for arm, seed in (("learned", 601), ("mix2", 801)):
        e = engine_ll(nx, T, seed, n_rep=n_rep)
        e.set_proposal(p)
        if arm == "mix2":
            e.set_proposal_mix(2)
        E1, S1 = replica_means(e, n_rep, 3000, 8000)
        acc = np.mean([e.series(r)["acceptance"].mean() for r in range(n_rep)])
        for name, a, b in [("E", E0, E1), ("S", S0, S1)]:
            se = np.sqrt(a.var(ddof=1) / n_rep + b.var(ddof=1) / n_rep)
            print("%s %s: plain %.6f  %s %.6f  se %.2g  z %+.2f  (acceptance %.3f)"
                  % (arm, name, a.mean(), arm, b.mean(), se, (b.mean() - a.mean()) / se, acc))
            assert abs(a.mean() - b.mean()) < 4 * se, (arm, name, a.mean(), b.mean(), se)
        e.close()
    plain.close()


EQUILIBRIUM_CASES = {
    # C2's physics: GHRL 1 : 0.5 : 1.5 slab with homeotropic anchoring W = 1.5 on both plates
    "ghrl_slab": (lambda: M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=[("homeotropic", 1.5, 0, 0)] * 2),
                  (12, 12, 8), 0.8),
    # C5's physics: pear slab, planar degenerate anchoring, dipolar field along z. The plain sweep follows every
    # rotation with an n -> -n trial; the learned proposal has none: it draws the new director with a random sign
    # (its density is even in n), so both orientations are proposed directly.
    "pear_field": (lambda: M.Model("pear", field_dir=(0, 0, 1), elecP=1.0, surfaces=[("fg", 1.0, 0, 0)] * 2),
                   (12, 12, 8), 0.5),
}


@pytest.mark.parametrize("case", sorted(EQUILIBRIUM_CASES))
def test_learned_sweep_keeps_the_equilibrium_of_c2_and_c5_physics(case):
    """<E>, <S> and, for the polar model, the polar order |sum n| / N of learned sweeps (untrained weights: any
    weights leave the distribution exact) against the plain sweep's, 8 replicas each, within 4 combined standard
    errors."""
    make_model, (nx, ny, nz), T = EQUILIBRIUM_CASES[case]
    n_rep = 8

    def run(learned, seed):
        reps = [M.Replica(nx, ny, nz, "slab", (1, 1, 0), T=T, seed=seed + r) for r in range(n_rep)]
        e = M.Engine(make_model(), reps, M.SCHED_CHECKER2)
        for r in range(n_rep):
            e.upload(r, rand_dirs(nx * ny * nz, seed + 100 * r, bias=1.5))
        if learned:
            e.set_proposal(perturbed_params(12))
        e.sweeps(800)
        e.clear_series()
        e.sweeps(3000, measure=True)
        out = []
        for r in range(n_rep):
            s = e.series(r)
            out.append((s["energy"].mean(), s["S"].mean(),
                        (np.linalg.norm(s["nsum"], axis=1) / s["n_valid"]).mean(), s["acceptance"].mean()))
        e.close()
        return np.array(out)

    plain, learned = run(False, 31), run(True, 71)
    assert learned[:, 3].mean() > 0.02  # the learned trials are accepted at all
    # The polar order is an equilibrium observable of the polar pear model only. GHRL is invariant under flipping
    # any single director, so its equilibrium has |sum n| / N ~ 0; the plain chain (small rotations, no flip trial)
    # keeps the polar order of its start, while the learned proposal's random sign samples both orientations.
    names = ["E", "S", "P"] if case == "pear_field" else ["E", "S"]
    if case != "pear_field":
        assert learned[:, 2].mean() < 0.1 < plain[:, 2].mean()
    for c, name in enumerate(names):
        a, b = plain[:, c], learned[:, c]
        se = np.sqrt(a.var(ddof=1) / n_rep + b.var(ddof=1) / n_rep)
        assert abs(a.mean() - b.mean()) < 4 * se + 1e-4, (case, name, a.mean(), b.mean(), se)


LEARNED_SHAPES = [
    # (potential, nx, ny, nz, geometry, periodic)
    ("ll", 64, 16, 20, "bulk", (1, 1, 1)),
    ("ll", 72, 22, 30, "bulk", (1, 1, 1)),    # ragged x and y tiles, several z segments
    ("ll", 30, 18, 26, "bulk", (0, 0, 0)),    # free everywhere
    ("ll", 2, 2, 2, "bulk", (1, 1, 1)),       # ghosts of ghosts
    ("ll", 6, 4, 4, "bulk", (1, 0, 1)),
    ("ghrl", 68, 20, 17, "slab", (1, 1, 0)),  # anchoring on both plates
    ("pear", 40, 12, 9, "slab", (0, 1, 0)),
]


@pytest.mark.parametrize("shape", LEARNED_SHAPES, ids=["%s-%dx%dx%d-%s-%s" % (s[0], s[1], s[2], s[3], s[4],
                                                                             "".join(map(str, s[5])))
                                                       for s in LEARNED_SHAPES])
def test_learned_passes_match_the_gathering_kernel(shape, monkeypatch):
    """The learned colour passes (planes in shared memory, one tcgen05 batch per plane) and the kernel that gathers
    each site's neighbours from global memory make every per-site computation alike, so they take the same
    decisions: identical directors and acceptance, observables equal up to the order of the sums."""
    pot, nx, ny, nz, geo, per = shape
    surf = {"slab": [("homeotropic", 1.2, 0, 0), ("fg", 0.6, 0, 0)]}.get(geo, [])
    if pot == "ghrl":
        model = M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=surf)
    elif pot == "pear":
        model = M.Model("pear", A=1.5, B1=0.09, C=0.3, surfaces=surf)
    else:
        model = M.Model("ll", surfaces=surf)
    params = perturbed_params(4)
    out = {}
    for kern in ("gather", "pass"):
        if kern == "gather":
            monkeypatch.setenv("MCL_LEARNED_KERNEL", "gather")
        else:
            monkeypatch.delenv("MCL_LEARNED_KERNEL", raising=False)
        e = M.Engine(model, [M.Replica(nx, ny, nz, geo, per, T=0.9, seed=21)], M.SCHED_CHECKER2)
        e.upload(0, rand_dirs(nx * ny * nz, 8))
        e.set_sweep_counter(17)
        e.set_proposal(params)
        e.sweeps(3, measure=True)
        out[kern] = (e.download(0), e.series(0))
        e.close()
    (a, sa), (b, sb) = out["gather"], out["pass"]
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(sa["acceptance"], sb["acceptance"])
    np.testing.assert_allclose(sa["energy"], sb["energy"], rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(sa["q"], sb["q"], rtol=0, atol=2e-7)
