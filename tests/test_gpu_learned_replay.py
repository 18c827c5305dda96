"""The learned Metropolis-Hastings sweep replayed decision by decision against the oracle (oracle/learned.py).

One learned sweep runs on the GPU from a known state at a known sweep counter; the same sweep is then replayed
site by site on the host, colour 0 from the initial state and colour 1 from the initial state with the GPU's
colour-0 results (the state each colour saw on the device):
  * the features of the site's neighbours, computed in FP32 with the kernel's fused multiply-adds,
  * the network outputs for those features from the tensor-core forward path the sweep kernels use (the network
    itself is checked against the oracle's forward pass in test_gpu_learned.py),
  * the head (axis mu, concentration kappa) and the site's Philox stream-1 block (counter (site, sweep, seed),
    the proposal's draws: mixture, Wood's w, azimuth, sign, acceptance),
  * the oracle's sampler (Wood's method with the 5 % uniform mixture and the random sign), the FP64 Lebwohl-Lasher
    site energies of the old and the proposed director, the symmetrised-vMF densities and the Hastings test
    u q(n') < exp(-dE / T) q(n).
Every decision must agree with the GPU's, except where the two sides are within rounding of the threshold (the
device works in FP32 with hardware exp/log/sin); every accepted director must equal the oracle's proposal to FP32
rounding of the sampler. Run for the colour-pass learned kernel (the default) and the gathering kernel."""
import numpy as np
import pytest

from helpers import M, O
from oracle import learned as L

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

PHILOX_KEY0, PHILOX_KEY1 = 0x694C634D, 0x30303242  # common.cuh: the key of stream s is (KEY0 + s, KEY1)
SHAPE = (12, 10, 8)
T = 0.9
SEED = 0x1234_5678_9ABC
SWEEP = 7
MARGIN = 1e-3  # log units: decisions this close to the threshold may go either way


def stream_block(seed, sweep, site, stream):
    ctr = [site & 0xFFFFFFFF, sweep & 0xFFFFFFFF, seed & 0xFFFFFFFF, ((seed >> 32) + (sweep >> 32)) & 0xFFFFFFFF]
    return O.philox(ctr, [(PHILOX_KEY0 + stream) & 0xFFFFFFFF, PHILOX_KEY1])


def u24(v):
    return (v >> 8) * 2.0 ** -24


def fma32(a, b, c):
    """float32 fused multiply-add: the float32 product is exact in double, one rounding of the sum to float32."""
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def features_f32(nb):
    """learned.cu site_features for one site (all weights 1: periodic lattice), in float32 with its FMAs."""
    f32 = np.float32
    mxx = mxy = mxz = myy = myz = mzz = f32(0.0)
    k = f32(0.0)
    for n in nb:
        ax, ay, az = f32(1.0) * n[0], f32(1.0) * n[1], f32(1.0) * n[2]
        mxx, mxy, mxz = fma32(ax, n[0], mxx), fma32(ax, n[1], mxy), fma32(ax, n[2], mxz)
        myy, myz, mzz = fma32(ay, n[1], myy), fma32(ay, n[2], myz), fma32(az, n[2], mzz)
        k = f32(k + f32(1.0))
    c = f32(1.0) / f32(6.0)
    return np.array([f32(fma32(1.5, mxx, f32(-0.5) * k) * c), f32(f32(1.5) * mxy * c), f32(f32(1.5) * mxz * c),
                     f32(fma32(1.5, myy, f32(-0.5) * k) * c), f32(f32(1.5) * myz * c),
                     f32(fma32(1.5, mzz, f32(-0.5) * k) * c), f32(T)], np.float32)


def neighbours(x, i, j, k):
    nx, ny, nz = SHAPE
    idx = lambda a, b, c: (a % nx) + nx * ((b % ny) + ny * (c % nz))  # noqa: E731
    return [x[idx(i + 1, j, k)], x[idx(i - 1, j, k)], x[idx(i, j + 1, k)], x[idx(i, j - 1, k)],
            x[idx(i, j, k + 1)], x[idx(i, j, k - 1)]]


def ll_energy(n, nb):
    return -1.5 * sum(float(np.dot(n, m)) ** 2 for m in nb)


def params(kappa_bias):
    rng = np.random.default_rng(21)
    p = L.init_params(5)
    p = p + 0.5 * rng.normal(size=p.size) * np.abs(p).mean()
    w1, b1, w2, b2, w3, b3 = L.unpack(p)
    b3 = b3.copy()
    b3[3] = kappa_bias  # the concentration's bias: proposals both accepted and rejected
    return L.pack([w1, b1, w2, b2, w3, b3]).astype(np.float32)


def network_outputs(p, feats):
    n = feats.shape[0]
    x = np.zeros((n, 8), np.float32)
    x[:, :7] = feats
    x[:, 7] = 1
    f = torch.from_numpy(x).cuda()
    out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    M.mlp_forward(p, f.data_ptr(), n, out.data_ptr(), tcgen05=True)
    return out.cpu().numpy().astype(np.float64)


def replay_colour(p, x_seen, colour):
    """Decisions of one colour on the state x_seen: dict site -> (accept, margin, proposal)."""
    nx, ny, nz = SHAPE
    sites, feats, nbs = [], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                if (i + j + k) % 2 != colour:
                    continue
                nb = neighbours(x_seen, i, j, k)
                sites.append(i + nx * (j + ny * k))
                feats.append(features_f32(nb))
                nbs.append(nb)
    o = network_outputs(p, np.array(feats))
    mu, kappa, _ = L.head(o, L.KAPPA_MAX)
    out = {}
    for s, site in enumerate(sites):
        u = stream_block(SEED, SWEEP, site, 1)
        n_old = x_seen[site].astype(np.float64)
        n_new = L.sample(mu[s:s + 1], kappa[s:s + 1], np.array([u24(u[0])]), np.array([u24(u[1])]),
                         np.array([u24(u[2])]), np.array([bool(u[0] & 1)]))[0]
        nb = [m.astype(np.float64) for m in nbs[s]]
        dE = ll_energy(n_new, nb) - ll_energy(n_old, nb)
        lq_old = L.log_q(n_old[None], mu[s:s + 1], kappa[s:s + 1])[0]
        lq_new = L.log_q(n_new[None], mu[s:s + 1], kappa[s:s + 1])[0]
        margin = np.log(max(u24(u[3]), 1e-300)) + lq_new - (-dE / T + lq_old)
        out[site] = (margin < 0, margin, n_new)
    return out


# kappa of a few, and kappa near 12, where e^{-2 kappa} is below FP32 resolution next to 1 (1 + expm1(-2 kappa) is
# then 0, and a density built from it loses its second term)
@pytest.mark.parametrize("kappa_bias", [2.5, 12.0])
@pytest.mark.parametrize("kernel", ["passes", "gather"])
def test_learned_sweep_replays_decision_by_decision(kernel, kappa_bias, monkeypatch):
    if kernel == "gather":
        monkeypatch.setenv("MCL_LEARNED_KERNEL", "gather")
    else:
        monkeypatch.delenv("MCL_LEARNED_KERNEL", raising=False)
    nx, ny, nz = SHAPE
    N = nx * ny * nz
    rng = np.random.default_rng(3)
    v = rng.normal(size=(N, 3))
    v[:, 2] += 1.2  # partly ordered, so the network's axis matters
    x0 = (v / np.linalg.norm(v, axis=1)[:, None]).astype(np.float32)
    p = params(kappa_bias)
    e = M.Engine(M.Model("ll"), [M.Replica(nx, ny, nz, T=T, seed=SEED)], M.SCHED_CHECKER2)
    e.upload(0, x0.reshape(-1))
    e.set_proposal(p)
    e.set_sweep_counter(SWEEP)
    e.sweeps(1)
    x1 = e.download(0).reshape(-1, 3)
    e.close()

    colour0 = replay_colour(p, x0, 0)
    x_half = x0.copy()
    for site in colour0:
        x_half[site] = x1[site]  # the state the colour-1 pass saw on the device
    colour1 = replay_colour(p, x_half, 1)

    accepted = mismatched = 0
    worst = 0.0
    for site, (acc, margin, n_new) in {**colour0, **colour1}.items():
        moved = bool(np.any(x1[site] != x0[site]))
        if moved != acc:
            assert abs(margin) < MARGIN, (site, moved, margin)
            mismatched += 1
            continue
        if moved:
            accepted += 1
            worst = max(worst, float(np.abs(x1[site] - n_new).max()))
    assert worst < 2e-5, worst
    assert mismatched <= 3, mismatched
    assert 0.01 * N < accepted < 0.95 * N, accepted  # both outcomes exercised


def philox_np(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 on arrays of counters (the oracle's mco_philox4x32_10, vectorised; checked against it below)."""
    mask = np.uint64(0xFFFFFFFF)
    c = [np.asarray(v, np.uint64) & mask for v in (c0, c1, c2, c3)]
    k0, k1 = np.uint64(k0), np.uint64(k1)
    for _ in range(10):
        p0, p1 = np.uint64(0xD2511F53) * c[0], np.uint64(0xCD9E8D57) * c[2]
        c = [((p1 >> np.uint64(32)) ^ c[1] ^ k0) & mask, p1 & mask, ((p0 >> np.uint64(32)) ^ c[3] ^ k1) & mask, p0 & mask]
        k0, k1 = (k0 + np.uint64(0x9E3779B9)) & mask, (k1 + np.uint64(0xBB67AE85)) & mask
    return c


def fixed_params(kappa_out):
    """Network weights 0: the output is the last bias, mu = z and kappa = softplus(kappa_out) at every site."""
    w1, b1, w2, b2, w3, b3 = L.unpack(L.init_params(3))
    zero = [np.zeros_like(a) for a in (w1, b1, w2, b2, w3)]
    return L.pack(zero + [np.array([0.0, 0.0, 1.0, kappa_out])]).astype(np.float32)


@pytest.mark.parametrize("kernel", ["passes", "gather"])
def test_fixed_proposal_replays_across_the_axis(kernel, monkeypatch):
    """A proposal fixed at mu = z with kappa = 9, from directors close to the xy-plane, so that t = mu.n is near 0
    where the density's two exponential terms are equal and e^{-2 kappa} lies below FP32 resolution next to 1: every
    decision of a 48^3 sweep against the FP64 Hastings test, to 1e-4 in log units. An error of 1-2 % in q at t = 0
    (what a density built from 1 + expm1(-2 kappa) has in FP32) flips several of these decisions."""
    if kernel == "gather":
        monkeypatch.setenv("MCL_LEARNED_KERNEL", "gather")
    else:
        monkeypatch.delenv("MCL_LEARNED_KERNEL", raising=False)
    n = 48
    N, Tf, seed, sweep = n ** 3, 1.0, 0x5EED_0F_F1C5, 11
    # the vectorised Philox against the oracle's
    ref = stream_block(seed, sweep, 12345, 1)
    got = philox_np([12345], [sweep], [seed & 0xFFFFFFFF], [seed >> 32], PHILOX_KEY0 + 1, PHILOX_KEY1)
    assert [int(v[0]) for v in got] == list(ref)
    rng = np.random.default_rng(8)
    phi = rng.uniform(0, 2 * np.pi, N)
    v = np.stack([np.cos(phi), np.sin(phi), 0.1 * rng.normal(size=N)], 1)
    x0 = (v / np.linalg.norm(v, axis=1)[:, None]).astype(np.float32)
    e = M.Engine(M.Model("ll"), [M.Replica(n, n, n, T=Tf, seed=seed)], M.SCHED_CHECKER2)
    e.upload(0, x0.reshape(-1))
    e.set_proposal(fixed_params(9.0))
    e.set_sweep_counter(sweep)
    e.sweeps(1)
    x1 = e.download(0).reshape(-1, 3)
    e.close()
    kappa = float(np.float32(np.log1p(np.exp(np.float32(9.0)))))
    site = np.arange(N)
    xi, yi, zi = site % n, (site // n) % n, site // (n * n)
    colour = (xi + yi + zi) % 2
    o = philox_np(site, np.full(N, sweep), np.full(N, seed & 0xFFFFFFFF), np.full(N, seed >> 32), PHILOX_KEY0 + 1,
                  PHILOX_KEY1)
    u = [(w >> np.uint64(8)).astype(np.float64) * 2.0 ** -24 for w in o]
    sign = (o[0] & np.uint64(1)) != 0
    mu = np.tile([0.0, 0.0, 1.0], (N, 1))
    kap = np.full(N, kappa)
    proposal = L.sample(mu, kap, u[0], u[1], u[2], sign)

    def energies(state, dirs):
        g = state.reshape(n, n, n, 3).astype(np.float64)  # (z, y, x)
        nb = [np.roll(g, s, axis=a).reshape(-1, 3) for a in (0, 1, 2) for s in (1, -1)]
        return -1.5 * sum(np.einsum("ij,ij->i", dirs, m) ** 2 for m in nb)

    seen = x0.copy()
    worst, mismatched, accepted = 0.0, 0, 0
    for c in (0, 1):
        if c == 1:
            seen[colour == 0] = x1[colour == 0]  # the state the colour-1 pass saw on the device
        sel = colour == c
        n_old = seen.astype(np.float64)
        dE = energies(seen, proposal) - energies(seen, n_old)
        lq = L.log_q(n_old, mu, kap) - L.log_q(proposal, mu, kap)
        with np.errstate(divide="ignore"):
            margin = np.log(u[3]) - (-dE / Tf + lq)
        acc = margin < 0
        moved = np.any(x1 != x0, axis=1)
        bad = sel & (moved != acc)
        assert np.all(np.abs(margin[bad]) < 1e-4), (c, np.sort(np.abs(margin[bad]))[-5:])
        mismatched += int(bad.sum())
        ok = sel & moved & acc
        accepted += int(ok.sum())
        worst = max(worst, float(np.abs(x1[ok] - proposal[ok]).max(initial=0)))
    assert mismatched <= 3, mismatched
    # many proposals lie close to the axis, where the sampler takes the tangential part from 1 - w itself
    # (sqrt(1 - w^2) from an FP32 w near 1 was off by up to 4e-5 here)
    assert worst < 2e-5, worst
    assert accepted > 0.01 * N, accepted
