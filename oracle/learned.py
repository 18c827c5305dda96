"""FP64 CPU oracle of the learned Metropolis-Hastings proposal (no counterpart in the reference).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA kernels in mclics_b200/csrc/learned.cu.
The product never imports this module.

What it restates (the algorithm the kernels implement, in plain numpy):
  features   per site, the neighbour Q-tensor sum  sum_j w_j (3 n_j n_j^T - I) / 2  divided by 6 (xx, xy, xz, yy,
             yz, zz) and the temperature T; the site's own director is not an input, so the proposal is an
             independence proposal given the neighbours.
  network    7 -> 64 -> 64 -> 4 with SiLU, weights [out][in]; operands rounded to BF16 (features, weights, hidden
             activations), products accumulated in FP32 by the kernels (here in FP64), biases FP32. The
             activation is evaluated as h + h tanh(h), h = z / 2, then rounded to BF16 (silu_bf16); its gradient
             is the exact SiLU derivative at z (straight through the rounding).
  head       axis mu = o[0:3] / |o[0:3]|, concentration kappa = clip(softplus(o[3]), KAPPA_MIN, kappa_max).
  proposal   q(n) = [ (1 - EPS) kappa cosh(kappa mu.n) / sinh(kappa) + EPS ] / (4 pi): an antipodally symmetrised
             von Mises-Fisher density mixed with EPS = 5 % uniform. Sampled by Wood's method (A. T. A. Wood,
             "Simulation of the von Mises Fisher distribution", Commun. Statist. 1994) with a random sign.
  accept     u < exp(-dE / T) q(n_old) / q(n_new)  (Hastings; q does not depend on the site's own director).
  training   loss = -mean log(4 pi q(n | features)) over samples (features, n) of equilibrated plain-sweep states,
             i.e. maximum likelihood of the site's local conditional distribution.
The LL site energy used by the tests is src/potential.cpp:28-31 of the reference summed over the six bonds.
"""
import numpy as np

N_IN, N_H, N_OUT = 7, 64, 4
EPS = 0.05
KAPPA_MIN = 1e-3
KAPPA_MAX = 500.0
N_PARAMS = N_H * N_IN + N_H + N_H * N_H + N_H + N_OUT * N_H + N_OUT


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def unpack(p):
    """Flat parameter vector (mcl_mlp order: w1[64][7], b1[64], w2[64][64], b2[64], w3[4][64], b3[4])."""
    p = np.asarray(p, dtype=np.float64)
    assert p.size == N_PARAMS
    o = 0
    out = []
    for shape in [(N_H, N_IN), (N_H,), (N_H, N_H), (N_H,), (N_OUT, N_H), (N_OUT,)]:
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1) for x in parts])


def init_params(seed=3):
    """Deterministic initial weights (uniform +-1/sqrt(fan_in), zero biases; kappa bias 1)."""
    rng = np.random.default_rng(seed)
    w1 = rng.uniform(-1, 1, (N_H, N_IN)) / np.sqrt(N_IN)
    w2 = rng.uniform(-1, 1, (N_H, N_H)) / np.sqrt(N_H)
    w3 = rng.uniform(-1, 1, (N_OUT, N_H)) / np.sqrt(N_H)
    b3 = np.zeros(N_OUT)
    b3[3] = 1.0
    return pack([w1, np.zeros(N_H), w2, np.zeros(N_H), w3, b3]).astype(np.float32).astype(np.float64)


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * sigmoid(z)


def silu_grad(z):
    s = sigmoid(z)
    return s * (1.0 + z * (1.0 - s))


def softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def features(nb, w, T):
    """nb: (n, 6, 3) neighbour directors, w: (n, 6) weights, T: scalar or (n,). Returns (n, 7)."""
    nb = np.asarray(nb, np.float64)
    w = np.asarray(w, np.float64)
    m = np.einsum("sj,sja,sjb->sab", w, nb, nb)
    k = w.sum(axis=1)
    q = 1.5 * m - 0.5 * k[:, None, None] * np.eye(3)[None]
    f = np.stack([q[:, 0, 0], q[:, 0, 1], q[:, 0, 2], q[:, 1, 1], q[:, 1, 2], q[:, 2, 2]], axis=1) / 6.0
    t = np.broadcast_to(np.asarray(T, np.float64), (f.shape[0],))
    return np.concatenate([f, t[:, None]], axis=1)


def _rounders(rounding):
    if rounding:
        return bf16, f32
    ident = lambda v: np.asarray(v, np.float64)  # noqa: E731
    return ident, ident


def silu_bf16(z):
    """The kernels' activation: z sigmoid(z) evaluated as h + h tanh(h) with h = z / 2, the result rounded to BF16
    (their tanh is the hardware approximation; here it is exact)."""
    h = 0.5 * np.asarray(z, np.float64)
    return bf16(h + h * np.tanh(h))


def forward(p, x, rounding=True):
    """Returns (out (n, 4), cache) with the BF16 rounding of the kernels (rounding=False: exact FP64, for
    finite-difference checks of the gradient formulas)."""
    r, rb = _rounders(rounding)
    act = silu_bf16 if rounding else silu
    w1, b1, w2, b2, w3, b3 = unpack(p)
    xb = r(x)
    z1 = xb @ r(w1).T + rb(b1)
    h1 = act(z1)
    z2 = h1 @ r(w2).T + rb(b2)
    h2 = act(z2)
    o = h2 @ r(w3).T + rb(b3)
    return o, (xb, z1, h1, z2, h2)


def head(o, kappa_max=KAPPA_MAX):
    a = o[:, :3]
    na = np.linalg.norm(a, axis=1)
    mu = np.where(na[:, None] > 1e-12, a / np.maximum(na, 1e-300)[:, None], np.array([0.0, 0.0, 1.0]))
    kraw = softplus(o[:, 3])
    kappa = np.clip(kraw, KAPPA_MIN, kappa_max)
    return mu, kappa, na


def g_of(t, kappa):
    """kappa cosh(kappa t) / sinh(kappa), overflow-free."""
    at = np.abs(t)
    return kappa * (np.exp(kappa * (at - 1.0)) + np.exp(-kappa * (at + 1.0))) / (-np.expm1(-2.0 * kappa))


def log_q(n, mu, kappa):
    """log(4 pi q(n)) of the mixture; n, mu: (m, 3)."""
    t = np.sum(n * mu, axis=1)
    return np.log((1.0 - EPS) * g_of(t, kappa) + EPS)


def loss_and_grad(p, x, n, kappa_max=KAPPA_MAX, rounding=True):
    """Mean loss -log(4 pi q(n | x)) and its gradient with respect to the parameters (straight through the BF16
    rounding of weights and activations, as the kernels do)."""
    r, _ = _rounders(rounding)
    w1, b1, w2, b2, w3, b3 = unpack(p)
    o, (xb, z1, h1, z2, h2) = forward(p, x, rounding)
    m = x.shape[0]
    a = o[:, :3]
    na = np.linalg.norm(a, axis=1)
    mu = a / na[:, None]
    kraw = softplus(o[:, 3])
    kappa = np.clip(kraw, KAPPA_MIN, kappa_max)
    t = np.sum(n * mu, axis=1)
    g = g_of(t, kappa)
    den = (1.0 - EPS) * g + EPS
    loss = -np.mean(np.log(den))
    # d(-log den) / dt and / dkappa
    dt = -(1.0 - EPS) * g * kappa * np.tanh(kappa * t) / den
    small = kappa < 0.1
    ik_minus_coth = np.where(small, -kappa / 3.0 + kappa ** 3 / 45.0,
                             1.0 / kappa - 1.0 / np.tanh(np.maximum(kappa, 1e-300)))
    dk = -(1.0 - EPS) * g * (ik_minus_coth + t * np.tanh(kappa * t)) / den
    dk = np.where((kraw > KAPPA_MIN) & (kraw < kappa_max), dk, 0.0)
    do = np.zeros_like(o)
    do[:, :3] = dt[:, None] * (n - t[:, None] * mu) / na[:, None]
    do[:, 3] = dk * sigmoid(o[:, 3])
    do /= m
    gw3 = do.T @ h2
    gb3 = do.sum(axis=0)
    dh2 = do @ r(w3)
    dz2 = dh2 * silu_grad(z2)
    gw2 = dz2.T @ h1
    gb2 = dz2.sum(axis=0)
    dh1 = dz2 @ r(w2)
    dz1 = dh1 * silu_grad(z1)
    gw1 = dz1.T @ xb
    gb1 = dz1.sum(axis=0)
    return loss, pack([gw1, gb1, gw2, gb2, gw3, gb3])


def sample(mu, kappa, u_mix, u_w, u_phi, sign_bit):
    """Wood's sampler with the mixture and the random sign, from given uniforms (the kernels' formulas)."""
    mu = np.asarray(mu, np.float64)
    kappa = np.asarray(kappa, np.float64)
    # vMF component: w = 1 + log(u + (1 - u) e^{-2 kappa}) / kappa
    w = 1.0 + np.log(u_w + (1.0 - u_w) * np.exp(-2.0 * kappa)) / kappa
    w = np.clip(w, -1.0, 1.0)
    uni = u_mix < EPS
    w = np.where(uni, 2.0 * u_w - 1.0, w)
    base = np.where(uni[:, None], np.array([0.0, 0.0, 1.0]), mu)
    e1, e2 = tangent_basis(base)
    r = np.sqrt(np.maximum(0.0, 1.0 - w * w))
    phi = 2.0 * np.pi * u_phi
    v = w[:, None] * base + r[:, None] * (np.cos(phi)[:, None] * e1 + np.sin(phi)[:, None] * e2)
    s = np.where(sign_bit & ~uni, -1.0, 1.0)
    return v * s[:, None]


def tangent_basis(mu):
    """Orthonormal e1, e2 perpendicular to unit mu (the kernels' construction)."""
    mu = np.asarray(mu, np.float64)
    helper = np.where(np.abs(mu[:, 0:1]) < 0.9, np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]))
    e1 = np.cross(mu, helper)
    e1 /= np.linalg.norm(e1, axis=1)[:, None]
    e2 = np.cross(mu, e1)
    return e1, e2


def tau_int(x, c=5.0):
    """Integrated autocorrelation time with Sokal's automatic window: the smallest W with W >= c tau(W), where
    tau(W) = 1/2 + sum_{t=1..W} rho(t), rho from the direct O(N W) sums (no FFT). Returns (tau, W)."""
    x = np.asarray(x, np.float64)
    n = x.size
    d = x - x.mean()
    var = np.dot(d, d) / n
    if var == 0:
        return 0.5, 0
    tau = 0.5
    for t in range(1, n):
        rho = np.dot(d[:-t], d[t:]) / (n * var)
        tau += rho
        if t >= c * tau:
            return tau, t
    return tau, n - 1
