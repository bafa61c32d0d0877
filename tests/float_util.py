"""Helpers for the float-descriptor tests: SIFT-like float descriptors that are not u/512, and
the reference's rules (tests/pyref.py) applied to a given score matrix, vectorised."""
import numpy as np

from v3dm import synth

f32 = np.float32


def float_descriptors(seed, nL, nR, planted=0.3):
    """Unit-length SIFT-like float descriptors (Gamma(0.6) -> normalise -> clamp 0.2 ->
    renormalise, not rounded), with noisy planted copies on the right."""
    rng = synth.rng_for(1000 + seed)

    def make(n):
        x = rng.gamma(0.6, 1.0, size=(n, 128))
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        np.minimum(x, 0.2, out=x)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        return x

    L = make(nL)
    n_p = int(planted * nR)
    src = rng.integers(0, nL, n_p)
    cp = np.abs(L[src] + rng.normal(0, 0.015, (n_p, 128)))
    cp /= np.linalg.norm(cp, axis=1, keepdims=True)
    R = np.concatenate([cp, make(nR - n_p)])[rng.permutation(nR)]
    return L.astype(np.float32), R.astype(np.float32)


def _side(M, ms, mr):
    n, m = M.shape
    if m == 0:
        return np.full(n, -1)
    arg = np.argmax(M, axis=1)
    mx = M[np.arange(n), arg]
    nxt = -np.sort(-M, axis=1)[:, 1] if m > 1 else np.full(n, f32(-1e30), np.float32)
    if mr < 0:
        return np.where(mx > f32(ms), arg, -1)
    nextDist = np.maximum(0.001, (f32(2.0) - f32(2.0) * nxt).astype(np.float64)).astype(np.float32)
    bestDist = (f32(2.0) - f32(2.0) * mx).astype(np.float32)
    ratio = (bestDist / nextDist).astype(np.float32)
    return np.where((mx > f32(ms)) & (ratio < f32(mr)), arg, -1)


def reference_pairs(S_lr, ms, mr):
    """Mutual ratio-test pairs of the reference (v3d_cudamatching.cu:133-210, :546-551) for the
    float32 score matrix S_lr[left, right]."""
    S = np.asarray(S_lr, np.float32)
    col = _side(S, ms, mr)      # per left, over rights
    row = _side(S.T, ms, mr)    # per right, over lefts
    out = [(k, col[k]) for k in range(S.shape[0]) if col[k] >= 0 and row[col[k]] == k]
    return np.array(out, np.int32).reshape(-1, 2)


def float_images(seed, n_images, n_min, n_max, exact=()):
    """An image set of float descriptors with shared tracks: synth.images' uint8 descriptors
    through synth.float_from_u8 (not u/512), except the images listed in 'exact', which keep
    u/512.  Returns (desc float32, counts, offsets)."""
    desc, counts, offs = synth.images(seed, n_images, n_min, n_max)
    out = synth.float_from_u8(desc, seed)
    for i in exact:
        out[offs[i]:offs[i + 1]] = desc[offs[i]:offs[i + 1]].astype(np.float32) / 512
    return out, counts, offs
