"""Training of the learned MH proposal on the GPU, from states of plain sweeps.

    import mclics_b200 as M
    from mclics_b200 import learned
    e = M.Engine(model, replicas)                  # plain proposal
    e.sweeps(500)                                  # thermalisation
    feat, dirs = learned.collect(e, snapshots=20, gap=10, per_snapshot=166_667, seed=3)
    params, losses = learned.train(feat, dirs, epochs=3, seed=3)
    e.set_proposal(params)                         # learned sweeps from here on

Samples are (features of a site's neighbours and T, the site's director) from equilibrated states
(mcl_extract_samples); the loss is -log(4 pi q(n | features)), i.e. maximum likelihood of the site's conditional
distribution given its neighbours (mcl_trainer_*: forward and backward kernels, Adam). torch only holds the device
buffers and shuffles the sample order.
"""
import math

import numpy as np

import mclics_b200 as M

N_H, N_IN, N_OUT = 64, 7, 4


def init_params(seed=3):
    """Initial weights: uniform +-1/sqrt(fan_in), zero biases, kappa bias 1."""
    rng = np.random.default_rng(seed)
    w1 = rng.uniform(-1, 1, (N_H, N_IN)) / math.sqrt(N_IN)
    w2 = rng.uniform(-1, 1, (N_H, N_H)) / math.sqrt(N_H)
    w3 = rng.uniform(-1, 1, (N_OUT, N_H)) / math.sqrt(N_H)
    b3 = np.zeros(N_OUT)
    b3[3] = 1.0
    p = np.concatenate([w1.ravel(), np.zeros(N_H), w2.ravel(), np.zeros(N_H), w3.ravel(), b3])
    assert p.size == M.N_MLP_PARAMS
    return p.astype(np.float32)


def collect(engine, snapshots, gap, per_snapshot, seed=3, replicas=None):
    """Samples from `snapshots` states `gap` plain sweeps apart, `per_snapshot` per replica and state. Returns
    device tensors (features n x 8, directors n x 3)."""
    import torch
    reps = list(range(engine.n)) if replicas is None else list(replicas)
    n = snapshots * len(reps) * per_snapshot
    feat = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    dirs = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    k = 0
    for s in range(snapshots):
        engine.sweeps(gap)
        for r in reps:
            engine.extract_samples(r, per_snapshot, seed * 1_000_003 + s * 1009 + r, feat[k:].data_ptr(),
                                   dirs[k:].data_ptr())
            k += per_snapshot
    return feat, dirs


def train(feat, dirs, epochs=3, batch=8192, lr=3e-3, lr_end=1e-4, seed=3, params=None):
    """Adam with a cosine learning-rate schedule over shuffled mini-batches. Returns (params, per-step losses)."""
    import torch
    n = feat.shape[0]
    if n < batch:
        raise ValueError("fewer samples (%d) than one batch (%d)" % (n, batch))
    p0 = init_params(seed) if params is None else M.mlp_params(params)
    t = M.Trainer(p0, batch)
    g = torch.Generator(device="cuda").manual_seed(seed)
    per_epoch = n // batch
    total = epochs * per_epoch
    losses = []
    try:
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device="cuda")
            for i in range(per_epoch):
                idx = perm[i * batch:(i + 1) * batch]
                fb, db = feat[idx].contiguous(), dirs[idx].contiguous()
                step = ep * per_epoch + i
                rate = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * step / max(1, total - 1)))
                losses.append(t.step(fb.data_ptr(), db.data_ptr(), batch, rate))
        out = t.params()
    finally:
        t.close()
    return out, np.array(losses)


def save(params, path):
    np.save(path, M.mlp_params(params))


def load(path):
    return M.mlp_params(np.load(path))
