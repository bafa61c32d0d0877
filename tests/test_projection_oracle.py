"""The CPU restatement of the learned projection (oracle/projection.py): its analytic
gradient agrees with central finite differences, and BF16 rounding is round-to-nearest-even."""
import numpy as np

from oracle import projection as P
from v3dm import synth


def _batch(seed, B):
    rng = synth.rng_for(seed)
    a = synth.sift_like(rng, B)
    p = synth.noisy_copy(rng, a, 8.0)
    return a, p


def test_gradient_matches_finite_differences():
    a, p = _batch(1, 12)
    w = P.init_params(3).astype(np.float64)
    T = 0.1
    loss, g = P.loss_grad(w, a, p, T, bf16=False)
    assert np.isfinite(loss) and g.shape == (P.N_PARAMS,)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(P.OFF_B1, 40, replace=False), P.OFF_B1 + rng.choice(P.N_HID, 10, replace=False),
                          P.OFF_W2 + rng.choice(P.N_OUT * P.N_HID, 30, replace=False),
                          P.OFF_B2 + rng.choice(P.N_OUT, 10, replace=False)])
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (P.loss_only(wp, a, p, T, bf16=False) - P.loss_only(wm, a, p, T, bf16=False)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_round_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265], np.float32)
    r = P.bf16_round(x)
    np.testing.assert_array_equal(r[:4], np.array([1.0, 1.0, 1.0 + 2 ** -7, 1.0 + 2 ** -6], np.float32))
    assert r[4] == -2.5 and abs(r[5] - 3.140625) < 1e-7


def test_loss_of_perfect_embedding_is_lower():
    """Matched pairs (noisy copies) give a lower loss than shuffled pairs."""
    a, p = _batch(2, 64)
    w = P.init_params(4)
    l_match, _ = P.loss_grad(w, a, p, 0.1)
    l_shuf, _ = P.loss_grad(w, a, p[::-1].copy(), 0.1)
    assert l_match < l_shuf
