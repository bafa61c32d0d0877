"""The candidate threshold T of the fused selection, checked by brute force on the host.

T must not exceed the smallest S that can pass the min-score test, and for every best score
S1 that can pass, the decision must be the same for every second value below T.  T is the
largest such value."""
import numpy as np
import pytest

f32 = np.float32


def _accept(s1, s2, ms, mr):
    s1 = s1.astype(np.float32)
    if mr < 0:
        return s1 > f32(ms)
    t = (f32(2.0) - f32(2.0) * np.float32(s2)).astype(np.float32)
    nextDist = np.maximum(0.001, t.astype(np.float64)).astype(np.float32)
    bestDist = (f32(2.0) - f32(2.0) * s1).astype(np.float32)
    ratio = (bestDist / nextDist).astype(np.float32)
    return (s1 > f32(ms)) & (ratio < f32(mr))


def _score(S):
    return (np.asarray(S, np.float32) * f32(2.0 ** -18)).astype(np.float32)


def _smin(ms):
    S = np.arange(0, 255 * 255 * 128 + 1)
    ok = np.flatnonzero(_score(S) > f32(ms))
    return int(ok[0]) if ok.size else 255 * 255 * 128 + 1


def _valid(T, ms, mr, gated):
    smin = _smin(ms)
    if T > smin:
        return False
    S1 = np.arange(smin, 2 ** 18 + 1)
    if S1.size == 0 or mr < 0:
        return True
    lo = _accept(_score(S1), f32(-1e30), ms, mr)
    hi_val = _score(T - 1) if T > 0 else (f32(-1e20) if gated else f32(-1e30))
    hi = _accept(_score(S1), hi_val, ms, mr)
    return bool(np.all(lo == hi))


@pytest.mark.parametrize("ms,mr", [(0.7, 0.8), (0.9, 0.8), (0.8, 0.6), (0.5, 0.95), (0.99, 0.99), (0.7, -1.0),
                                   (-0.3, 0.8), (0.0, 0.5), (0.7, 0.0), (0.7, 1.5)])
@pytest.mark.parametrize("gated", [False, True])
def test_threshold_is_valid_and_maximal(v3dm_mod, ms, mr, gated):
    T = v3dm_mod.candidate_threshold(ms, mr, gated)
    smin = _smin(ms)
    assert 0 <= T <= smin
    assert _valid(T, ms, mr, gated)
    if T < smin:
        assert not _valid(T + 1, ms, mr, gated)


def test_threshold_for_the_benchmark_parameters(v3dm_mod):
    # c = 1 - (1 - 0.7)/0.8 = 0.625 of 2^18
    T = v3dm_mod.candidate_threshold(0.7, 0.8, False)
    assert abs(T - 0.625 * 2 ** 18) <= 2


def test_threshold_nan_and_unsupported(v3dm_mod):
    T = v3dm_mod.candidate_threshold(float("nan"), 0.8, False)
    assert T == 255 * 255 * 128 + 1
    with pytest.raises(v3dm_mod.V3DMError) as e:
        v3dm_mod.candidate_threshold(-1.0, 1e-35, True)
    assert e.value.status == v3dm_mod.ERR_UNSUPPORTED


# ---- float candidate threshold of the BF16 hi/lo path ------------------------------------
@pytest.mark.parametrize("ms,mr", [(0.7, 0.8), (0.9, 0.8), (0.8, 0.6), (0.5, 0.95), (0.99, 0.99), (0.7, -1.0),
                                   (-0.3, 0.8), (0.0, 0.5), (0.7, 0.0), (0.7, 1.5)])
def test_float_threshold_is_valid_and_tight(v3dm_mod, ms, mr):
    Tf = f32(v3dm_mod.float_threshold(ms, mr))
    s1min = np.nextafter(f32(ms), f32(np.inf))
    assert Tf <= s1min
    rng = np.random.default_rng(0)
    s1 = np.concatenate([s1min + np.arange(0, 4096, dtype=np.float32) * np.spacing(s1min),
                         rng.uniform(float(s1min), 2.5, 20000).astype(np.float32)]).astype(np.float32)
    below = np.nextafter(Tf, f32(-np.inf))
    for s2 in (below, f32(-1e20), Tf - f32(0.25), rng.uniform(min(-1.0, float(below) - 1.0), float(below), 1).astype(np.float32)[0]):
        if s2 >= Tf:
            continue
        np.testing.assert_array_equal(_accept(s1, s2, ms, mr), _accept(s1, f32(-1e30), ms, mr))
    if Tf < s1min:  # tight: a second value of Tf changes the decision of the weakest best
        assert _accept(np.array([s1min]), Tf, ms, mr)[0] != _accept(np.array([s1min]), f32(-1e30), ms, mr)[0]


def test_float_threshold_for_the_benchmark_parameters(v3dm_mod):
    assert abs(v3dm_mod.float_threshold(0.7, 0.8) - 0.625) < 1e-6
