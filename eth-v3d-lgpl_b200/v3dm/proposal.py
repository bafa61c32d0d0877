"""Training pipeline of the learned candidate proposal.

1. Mine matched descriptor pairs: exhaustive batched matching (BatchMatching.match) of
   held-out images; every mutual ratio-test match (l, r) gives an (anchor, positive) pair.
2. Train the 128 -> 64 -> 32 projection (Projection.train_step: hand-written forward,
   InfoNCE loss, backward and Adam kernels) on random minibatches of those pairs.
3. Fit C cells: spherical k-means of the trained embeddings of the held-out descriptors.
Matching then uses BatchMatching.match_proposal(projection, probes, ...), with exhaustive
matching (BatchMatching.match) as the reference and fallback.
"""
from __future__ import annotations

import numpy as np


def mine_pairs(desc: np.ndarray, offsets: np.ndarray, pairs: np.ndarray, triples: np.ndarray):
    """(anchors, positives) uint8 arrays from exhaustive-match triples (pair, left, right)."""
    li = pairs[triples[:, 0], 0]
    ri = pairs[triples[:, 0], 1]
    a = desc[offsets[li] + triples[:, 1]]
    p = desc[offsets[ri] + triples[:, 2]]
    return np.ascontiguousarray(a), np.ascontiguousarray(p)


def train(projection, anchors: np.ndarray, positives: np.ndarray, steps: int = 400, batch: int = 2048,
          temperature: float = 0.05, lr: float = 2e-3, seed: int = 0, device: int = 0):
    """Adam on random minibatches; returns the per-step losses of every 50th step."""
    import torch
    dev = torch.device("cuda", device)
    da = torch.from_numpy(anchors).to(dev)
    dp = torch.from_numpy(positives).to(dev)
    n = anchors.shape[0]
    batch = min(batch, n)
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    for step in range(steps):
        idx = torch.randperm(n, generator=g)[:batch].to(dev)
        xa, xp = da[idx].contiguous(), dp[idx].contiguous()
        want = step % 50 == 0 or step == steps - 1
        loss = projection.train_step(xa.data_ptr(), xp.data_ptr(), batch, temperature, lr, want_loss=want)
        if want:
            losses.append((step, loss))
        del xa, xp
    torch.cuda.synchronize(dev)
    return losses


def fit_cells(z: np.ndarray, n_cells: int, iters: int = 25, seed: int = 0) -> np.ndarray:
    """Spherical k-means of unit vectors z (n x 32): unit centroids (n_cells x 32).  Seeded
    with k-means++ over a subsample; empty cells are re-seeded from the worst-served points."""
    rng = np.random.default_rng(seed)
    z = np.asarray(z, np.float32)
    sample = z[rng.choice(z.shape[0], min(z.shape[0], 200_000), replace=False)]
    cent = np.empty((n_cells, z.shape[1]), np.float32)
    cent[0] = sample[rng.integers(sample.shape[0])]
    best = sample @ cent[0]
    for c in range(1, n_cells):
        d = np.maximum(1.0 - best, 0.0) ** 2
        cent[c] = sample[rng.choice(sample.shape[0], p=d / d.sum())] if d.sum() > 0 else sample[rng.integers(sample.shape[0])]
        best = np.maximum(best, sample @ cent[c])
    for _ in range(iters):
        s = sample @ cent.T
        a = np.argmax(s, axis=1)
        new = np.zeros_like(cent)
        np.add.at(new, a, sample)
        norm = np.linalg.norm(new, axis=1)
        empty = norm < 1e-6
        if empty.any():
            worst = np.argsort(s[np.arange(sample.shape[0]), a])[: int(empty.sum())]
            new[empty] = sample[worst]
            norm[empty] = np.linalg.norm(new[empty], axis=1)
        cent = (new / norm[:, None]).astype(np.float32)
    return cent


def recall(exhaustive: np.ndarray, proposal: np.ndarray):
    """(recall, precision) of proposal triples against exhaustive triples."""
    e = {tuple(t) for t in exhaustive.tolist()}
    p = {tuple(t) for t in proposal.tolist()}
    hit = len(e & p)
    return hit / max(1, len(e)), hit / max(1, len(p))
