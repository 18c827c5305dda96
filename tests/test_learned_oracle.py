"""The FP64 oracle of the learned proposal, checked on its own: analytic gradients against central finite
differences, the proposal density's normalisation on the sphere, Wood's sampler against that density, and the
windowed tau_int against the exact value of an AR(1) process."""
import numpy as np

from oracle import learned as L


def batch(m, seed):
    rng = np.random.default_rng(seed)
    nb = rng.normal(size=(m, 6, 3))
    nb[:, :, 2] += 2.0
    nb /= np.linalg.norm(nb, axis=2)[:, :, None]
    x = L.features(nb, np.ones((m, 6)), rng.uniform(0.3, 1.2, m))
    n = rng.normal(size=(m, 3))
    n[:, 2] += 2.0
    n /= np.linalg.norm(n, axis=1)[:, None]
    return x, n


def test_gradient_matches_finite_differences():
    x, n = batch(64, 1)
    p = L.init_params(3)
    loss, g = L.loss_and_grad(p, x, n, rounding=False)
    rng = np.random.default_rng(7)
    idx = rng.choice(L.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [L.N_PARAMS - 1, L.N_PARAMS - 2, 0]])  # kappa bias, an axis bias, w1[0][0]
    h = 1e-6
    for i in idx:
        e = np.zeros(L.N_PARAMS)
        e[i] = h
        lp, _ = L.loss_and_grad(p + e, x, n, rounding=False)
        lm, _ = L.loss_and_grad(p - e, x, n, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_density_is_normalised():
    # q depends on t = mu.n only, so its integral over the sphere is 2 pi * int_{-1}^{1} q dt
    t = np.linspace(-1, 1, 200001)
    for kappa in [1e-3, 0.05, 1.0, 7.5, 60.0, 500.0]:
        q = np.exp(L.log_q(np.stack([np.zeros_like(t), np.zeros_like(t), t], 1), np.array([[0, 0, 1.0]]),
                           np.full(t.shape, kappa))) / (4 * np.pi)
        assert abs(2 * np.pi * np.trapezoid(q, t) - 1.0) < 1e-5, kappa  # trapezoid error ~2e-6 at kappa 500


def test_sampler_matches_density():
    rng = np.random.default_rng(5)
    m = 400000
    mu = rng.normal(size=(1, 3))
    mu /= np.linalg.norm(mu)
    for kappa in [0.5, 8.0, 80.0]:
        v = L.sample(np.repeat(mu, m, 0), np.full(m, kappa), rng.random(m), rng.random(m), rng.random(m),
                     rng.random(m) < 0.5)
        assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-12)
        t = v @ mu[0]
        hist, edges = np.histogram(t, bins=40, range=(-1, 1))
        tt = np.linspace(-1, 1, 40001)
        pdf = np.exp(L.log_q(np.stack([np.zeros_like(tt), np.zeros_like(tt), tt], 1), np.array([[0, 0, 1.0]]),
                             np.full(tt.shape, kappa))) / 2.0  # density of t
        cdf = np.concatenate([[0], np.cumsum((pdf[1:] + pdf[:-1]) / 2 * np.diff(tt))])
        expect = m * np.diff(np.interp(edges, tt, cdf))
        chi2 = np.sum((hist - expect) ** 2 / np.maximum(expect, 1e-9))
        assert chi2 < 40 + 4 * np.sqrt(80), (kappa, chi2)  # 39 degrees of freedom, generous bound
        # the azimuth about mu is uniform
        e1, e2 = L.tangent_basis(mu)
        phi = np.arctan2(v @ e2[0], v @ e1[0])
        h2, _ = np.histogram(phi, bins=16, range=(-np.pi, np.pi))
        assert np.max(np.abs(h2 / (m / 16) - 1)) < 0.03


def test_tau_int_of_ar1():
    rng = np.random.default_rng(11)
    for phi in [0.0, 0.5, 0.9]:
        n = 200000
        e = rng.normal(size=n)
        x = np.empty(n)
        x[0] = e[0]
        for i in range(1, n):
            x[i] = phi * x[i - 1] + e[i]
        tau, w = L.tau_int(x)
        exact = (1 + phi) / (2 * (1 - phi))
        assert abs(tau - exact) < 0.05 * exact + 0.02, (phi, tau, exact, w)


def test_fft_tau_int_matches_direct_sums():
    from mclics_b200 import analysis as A
    rng = np.random.default_rng(3)
    for phi in [0.0, 0.7, 0.97]:
        n = 20000
        e = rng.normal(size=n)
        x = np.empty(n)
        x[0] = e[0]
        for i in range(1, n):
            x[i] = phi * x[i - 1] + e[i]
        t_ref, w_ref = L.tau_int(x)
        t, w = A.tau_int(x)
        assert w == w_ref and abs(t - t_ref) < 1e-9 * max(1.0, t_ref), (phi, t, t_ref, w, w_ref)


def test_block_error_matches_the_exact_error_of_ar1_means():
    """Batch-means error of AR(1) series against the exact standard error of their mean,
    sqrt(var / N * (1 + phi) / (1 - phi)), over 200 series (the estimate itself scatters by ~1/sqrt(2 (B - 1)))."""
    from mclics_b200 import analysis as A
    rng = np.random.default_rng(5)
    phi, n, reps = 0.9, 32000, 200
    e = rng.normal(size=(reps, n))
    x = np.empty_like(e)
    x[:, 0] = e[:, 0] / np.sqrt(1 - phi ** 2)
    for i in range(1, n):
        x[:, i] = phi * x[:, i - 1] + e[:, i]
    exact = np.sqrt(1 / (1 - phi ** 2) / n * (1 + phi) / (1 - phi))
    est = np.array([A.block_error(s, 16) for s in x])
    assert abs(np.sqrt((est ** 2).mean()) / exact - 1) < 0.05
    # and the spread of the 200 means agrees with both
    assert abs(x.mean(axis=1).std(ddof=1) / exact - 1) < 0.15
