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


def params():
    rng = np.random.default_rng(21)
    p = L.init_params(5)
    p = p + 0.5 * rng.normal(size=p.size) * np.abs(p).mean()
    w1, b1, w2, b2, w3, b3 = L.unpack(p)
    b3 = b3.copy()
    b3[3] = 2.5  # a concentrated proposal (kappa of a few), so rotations are both accepted and rejected
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


@pytest.mark.parametrize("kernel", ["passes", "gather"])
def test_learned_sweep_replays_decision_by_decision(kernel, monkeypatch):
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
    p = params()
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
    assert 0.05 * N < accepted < 0.95 * N, accepted  # both outcomes exercised
