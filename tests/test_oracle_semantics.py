"""The C oracle against a literal Python restatement of the reference kernels (CPU only)."""
import numpy as np
import pytest

import pyref
from v3dm import synth


def _case(seed, nL, nR, dup=0):
    rng = np.random.default_rng(seed)
    L, R, _ = synth.pair(seed, nL, nR)
    if dup and nR > 2:
        # exact duplicates in R make ties: same score, ratio 1
        for _ in range(dup):
            a, b = rng.integers(0, nR, 2)
            R[b] = R[a]
    return L, R


@pytest.mark.parametrize("seed,nL,nR", [(0, 1, 1), (1, 5, 7), (2, 31, 33), (3, 64, 32), (4, 33, 96), (5, 0, 8)])
@pytest.mark.parametrize("ms,mr", [(0.7, 0.8), (0.9, 0.8), (0.5, 0.95), (0.7, -1.0), (-0.5, 0.8)])
def test_putative_matches_pyref(oracle_mod, seed, nL, nR, ms, mr):
    L, R = _case(seed, nL, nR, dup=3)
    got, col, row = oracle_mod.match(L, R, ms, mr, with_sides=True)
    if nL == 0 or nR == 0:
        assert got.shape == (0, 2)
        return
    exp, ecol, erow = pyref.match(L, R, ms, mr)
    np.testing.assert_array_equal(got, exp)
    np.testing.assert_array_equal(col, ecol)
    np.testing.assert_array_equal(row, erow)


def _positions(seed, n, w=640, h=480):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(0, w, n), rng.uniform(0, h, n)], 1).astype(np.float32)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_guided_matches_pyref(oracle_mod, seed):
    L, R, lp, rp, F, _ = synth.stereo(seed, 48, 40, width=640, height=480)
    H = np.array([[1.01, 0.02, 3.0], [-0.01, 0.99, -2.0], [1e-5, -2e-5, 1.0]])
    for gates in ([("F", F, 2.0)], [("H", H, 40.0)], [("F", F, 2.0), ("H", H, 200.0)]):
        got = oracle_mod.match(L, R, 0.7, 0.8, gates=gates, lpos=lp, rpos=rp)
        exp, _, _ = pyref.match(L, R, 0.7, 0.8, gates=gates, lpos=lp, rpos=rp)
        np.testing.assert_array_equal(got, exp)


def test_known_answers(oracle_mod):
    base = synth.sift_like(synth.rng_for(7), 4)
    L = base[:2].copy()
    # right 0 = left 0 exactly, right 1 = left 0 exactly (tie), right 2 = left 1 exactly
    R = np.stack([base[0], base[0], base[1], base[3]])
    got, col, row = oracle_mod.match(L, R, 0.7, 0.8, with_sides=True)
    # left 0 has a tie between rights 0 and 1: ratio 1 -> rejected
    assert col[0] == -1
    # left 1 matches right 2 (score ~1, next far below)
    assert col[1] == 2 and row[2] == 1
    np.testing.assert_array_equal(got, np.array([[1, 2]], np.int32))
    # without the ratio test the tie resolves to the first index
    got, col, row = oracle_mod.match(L, R, 0.7, -1.0, with_sides=True)
    assert col[0] == 0 and row[0] == 0 and row[1] == 0
    np.testing.assert_array_equal(got, np.array([[0, 0], [1, 2]], np.int32))


def test_empty_and_masked(oracle_mod):
    L, R = _case(11, 16, 16)
    assert oracle_mod.match(L[:0], R, 0.7, 0.8).shape == (0, 2)
    assert oracle_mod.match(L, R[:0], 0.7, 0.8).shape == (0, 2)
    lp = _positions(1, 16)
    rp = _positions(2, 16)
    F = np.array([[0, 0, 0], [0, 0, -1.0], [0, 1.0, 0]])  # q.y == p.y lines; threshold 0 masks all
    got = oracle_mod.match(L, R, 0.7, 0.8, gates=[("F", F, 0.0)], lpos=lp, rpos=rp)
    assert got.shape == (0, 2)


def test_reference_truncation(oracle_mod):
    # .cu:444-460 and .cu:493-519: round down to a multiple of 32, clamp to nMax
    assert oracle_mod.ref_feature_count(100, 96) == 96
    assert oracle_mod.ref_feature_count(95, 4096) == 64
    assert oracle_mod.ref_feature_count(31, 4096) == 0


def test_threads_do_not_change_result(oracle_mod):
    L, R, _ = synth.pair(5, 700, 900)
    a = oracle_mod.match(L, R, 0.7, 0.8, threads=1)
    b = oracle_mod.match(L, R, 0.7, 0.8, threads=7)
    np.testing.assert_array_equal(a, b)


def test_one_score_pass_equals_separate_calls():
    """match_calls (putative and compounding guided calls from one score computation, as the
    reference masks its stored matrix) equals separate oracle calls."""
    import numpy as np
    from oracle import oracle
    from v3dm import synth
    L, R, lp, rp, F, _ = synth.stereo(3, 900, 1000)
    H = np.eye(3)
    H[0, 2] = 5.0
    calls = [[], [("F", F, 2.0)], [("F", F, 2.0), ("H", H, 400.0)]]
    got = oracle.match_calls(L, R, 0.7, 0.8, calls, lpos=lp, rpos=rp, threads=3)
    for g, c in zip(got, calls):
        exp = oracle.match(L, R, 0.7, 0.8, gates=c, lpos=lp, rpos=rp)
        assert np.array_equal(g, exp)
    assert got[0].shape[0] > got[2].shape[0] > 0
