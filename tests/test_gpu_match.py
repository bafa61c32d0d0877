"""Parity of the CUDA matcher (through the C ABI) with the oracle: bit-exact pairs."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu

KERNELS = ["simt", "tcgen05"]


def _kernel_id(v3dm, name):
    return v3dm.KERNEL_SIMT if name == "simt" else v3dm.KERNEL_TCGEN05


@pytest.fixture(params=KERNELS)
def make_matcher(request, v3dm_mod):
    made = []

    def make(nL, nR, guided=False):
        m = v3dm_mod.SIFTMatching(0, _kernel_id(v3dm_mod, request.param))
        m.allocate(nL, nR, guided)
        made.append(m)
        return m

    yield make
    for m in made:
        m.close()


def _run(m, L, R, ms, mr):
    m.set_left_features(L)
    m.set_right_features(R)
    return m.find_putative_matches(ms, mr)


@pytest.mark.parametrize("seed", range(4))
def test_pair_4096_bit_exact(make_matcher, oracle_mod, seed):
    L, R, _ = synth.pair(seed)
    m = make_matcher(4096, 4096)
    got = _run(m, L, R, synth.MIN_SCORE, synth.MIN_RATIO)
    exp = oracle_mod.match(L, R, synth.MIN_SCORE, synth.MIN_RATIO)
    assert exp.shape[0] > 800
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("nL,nR", [(1, 1), (1, 300), (31, 33), (127, 129), (128, 256), (300, 1000), (1000, 257),
                                   (4095, 4097), (0, 5), (5, 0)])
def test_ragged_sizes(make_matcher, oracle_mod, nL, nR):
    L, R, _ = synth.pair(100 + nL, nL, nR)
    m = make_matcher(max(nL, 1), max(nR, 1))
    got = _run(m, L, R, 0.7, 0.8)
    exp = oracle_mod.match(L, R, 0.7, 0.8)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("ms,mr", [(0.9, 0.8), (0.5, 0.95), (0.7, -1.0), (0.6, 1.2), (-0.5, 0.8), (0.95, 0.5)])
def test_parameters(make_matcher, oracle_mod, ms, mr):
    L, R, _ = synth.pair(21, 1500, 1700)
    m = make_matcher(1500, 1700)
    got = _run(m, L, R, ms, mr)
    exp = oracle_mod.match(L, R, ms, mr)
    np.testing.assert_array_equal(got, exp)


def test_ties_and_duplicates(make_matcher, oracle_mod):
    L, R, _ = synth.pair(33, 900, 1100)
    rng = np.random.default_rng(3)
    for _ in range(100):  # exact duplicate rights and lefts: equal scores, ratio 1
        a, b = rng.integers(0, 1100, 2)
        R[b] = R[a]
        c, d = rng.integers(0, 900, 2)
        L[d] = L[c]
    R[:50] = L[:50]  # perfect copies
    m = make_matcher(900, 1100)
    for mr in (0.8, -1.0):
        got = _run(m, L, R, 0.7, mr)
        exp = oracle_mod.match(L, R, 0.7, mr)
        np.testing.assert_array_equal(got, exp)


def test_repeated_calls_reset_state(make_matcher, oracle_mod):
    m = make_matcher(2048, 2048)
    for seed in (5, 6, 5):
        L, R, _ = synth.pair(seed, 2048, 2000)
        got = _run(m, L, R, 0.7, 0.8)
        np.testing.assert_array_equal(got, oracle_mod.match(L, R, 0.7, 0.8))
        got2 = m.find_putative_matches(0.7, 0.8)
        np.testing.assert_array_equal(got2, got)


def test_float_inputs(make_matcher, oracle_mod, v3dm_mod):
    L, R, _ = synth.pair(8, 700, 800)
    m = make_matcher(700, 800)
    got = _run(m, L.astype(np.float32) / 512, R.astype(np.float32) / 512, 0.7, 0.8)
    np.testing.assert_array_equal(got, oracle_mod.match(L, R, 0.7, 0.8))
    bad = L.astype(np.float32) / 512
    bad[3, 7] += 1e-4
    if m.kernel == v3dm_mod.KERNEL_SIMT:
        with pytest.raises(v3dm_mod.V3DMError) as e:
            m.set_left_features(bad)
        assert e.value.status == v3dm_mod.ERR_NOT_U8
    else:  # the tcgen05 handle takes the BF16 hi/lo path for such floats
        m.set_left_features(bad)
        assert m.find_putative_matches(0.7, 0.8).shape[0] > 0
        bad[0, 0] = np.nan
        with pytest.raises(v3dm_mod.V3DMError) as e:
            m.set_left_features(bad)
        assert e.value.status == v3dm_mod.ERR_ARG


def test_size_errors(make_matcher, v3dm_mod):
    m = make_matcher(100, 100)
    L, R, _ = synth.pair(1, 101, 10)
    with pytest.raises(v3dm_mod.V3DMError) as e:
        m.set_left_features(L)
    assert e.value.status == v3dm_mod.ERR_SIZE


@pytest.mark.parametrize("seed", [1, 2])
def test_guided_epipolar(make_matcher, oracle_mod, seed):
    L, R, lp, rp, F, _ = synth.stereo(seed, 3000, 2800)
    m = make_matcher(3000, 2800, guided=True)
    m.set_left_features(L)
    m.set_right_features(R)
    put = m.find_putative_matches(0.7, 0.8)
    np.testing.assert_array_equal(put, oracle_mod.match(L, R, 0.7, 0.8))
    got = m.run_guided_matching(F, 2.0, lp, rp, 0.7, 0.8)
    exp = oracle_mod.match(L, R, 0.7, 0.8, gates=[("F", F, 2.0)], lpos=lp, rpos=rp)
    assert exp.shape[0] > put.shape[0] * 0.5
    np.testing.assert_array_equal(got, exp)


def test_guided_homography_and_compounding(make_matcher, oracle_mod):
    L, R, lp, rp, F, _ = synth.stereo(4, 2000, 2100)
    H = np.array([[1.0, 0.01, 25.0], [0.0, 1.0, 3.0], [0.0, 0.0, 1.0]])
    m = make_matcher(2000, 2100, guided=True)
    m.set_left_features(L)
    m.set_right_features(R)
    m.find_putative_matches(0.7, 0.8)
    got1 = m.run_guided_homography_matching(H, 300.0, lp, rp, 0.7, 0.8)
    exp1 = oracle_mod.match(L, R, 0.7, 0.8, gates=[("H", H, 300.0)], lpos=lp, rpos=rp)
    np.testing.assert_array_equal(got1, exp1)
    # a second guided call compounds with the first, as the in-place masking does
    got2 = m.run_guided_matching(F, 4.0, lp, rp, 0.7, 0.8)
    exp2 = oracle_mod.match(L, R, 0.7, 0.8, gates=[("H", H, 300.0), ("F", F, 4.0)], lpos=lp, rpos=rp)
    np.testing.assert_array_equal(got2, exp2)
    # putative clears the gates
    np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), oracle_mod.match(L, R, 0.7, 0.8))


def test_guided_reuses_putative_pass(make_matcher, oracle_mod):
    """A guided call after a putative call on the same features reuses that call's pass A
    (records and bounds) when its minimum score is the same and its threshold allows it, and
    recomputes otherwise; new features drop the stored pass.  Every result is the reference's."""
    L, R, lp, rp, F, _ = synth.stereo(9, 2500, 2600)
    m = make_matcher(2600, 2600, guided=True)
    m.set_left_features(L)
    m.set_right_features(R)
    for ms, mr in [(0.7, 0.8), (0.7, 0.95), (0.7, 0.6), (0.75, 0.8), (0.6, -1.0)]:
        np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), oracle_mod.match(L, R, 0.7, 0.8))
        got = m.run_guided_matching(F, 2.0, lp, rp, ms, mr)
        exp = oracle_mod.match(L, R, ms, mr, gates=[("F", F, 2.0)], lpos=lp, rpos=rp)
        np.testing.assert_array_equal(got, exp, err_msg=f"minScore {ms} ratio {mr}")
    # new left features: the next guided call cannot use the stored pass
    L2, R2, lp2, rp2, F2, _ = synth.stereo(10, 2400, 2600)
    m.find_putative_matches(0.7, 0.8)
    m.set_left_features(L2)
    m.set_right_features(R2)
    got = m.run_guided_matching(F2, 2.0, lp2, rp2, 0.7, 0.8)
    np.testing.assert_array_equal(got, oracle_mod.match(L2, R2, 0.7, 0.8, gates=[("F", F2, 2.0)], lpos=lp2,
                                                        rpos=rp2))


def test_stereo_16384_guided(make_matcher, oracle_mod):
    """The 16384 x 16384 guided workload: putative and guided pairs bit-exact."""
    L, R, lp, rp, F, truth = synth.stereo(1)
    m = make_matcher(16384, 16384, guided=True)
    m.set_left_features(L)
    m.set_right_features(R)
    put = m.find_putative_matches(synth.MIN_SCORE, synth.MIN_RATIO)
    np.testing.assert_array_equal(put, oracle_mod.match(L, R, synth.MIN_SCORE, synth.MIN_RATIO))
    got = m.run_guided_matching(F, 2.0, lp, rp, synth.MIN_SCORE, synth.MIN_RATIO)
    exp = oracle_mod.match(L, R, synth.MIN_SCORE, synth.MIN_RATIO, gates=[("F", F, 2.0)], lpos=lp, rpos=rp)
    np.testing.assert_array_equal(got, exp)
    # size-independent property: guided pairs agree with the planted geometry
    assert np.mean(truth[got[:, 1]] == got[:, 0]) > 0.99


@pytest.mark.parametrize("nL,nR", [(300, 1000), (4095, 4097), (257, 63)])
def test_every_tile_config(v3dm_mod, oracle_mod, nL, nR):
    L, R, lp, rp, F, _ = synth.stereo(7 + nL, nL, nR)
    exp_put = oracle_mod.match(L, R, 0.7, 0.8)
    exp_gui = oracle_mod.match(L, R, 0.7, 0.8, gates=[("F", F, 2.0)], lpos=lp, rpos=rp)
    with v3dm_mod.SIFTMatching(0, v3dm_mod.KERNEL_TCGEN05) as m:
        m.allocate(nL, nR, True)
        m.set_left_features(L)
        m.set_right_features(R)
        for cfg in range(m.num_configs()):
            m.set_config(cfg)
            np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), exp_put, err_msg=f"config {cfg}")
            np.testing.assert_array_equal(m.run_guided_matching(F, 2.0, lp, rp, 0.7, 0.8), exp_gui,
                                          err_msg=f"config {cfg}")


def test_autotune_keeps_results(v3dm_mod, oracle_mod):
    L, R, _ = synth.pair(3, 3000, 3500)
    with v3dm_mod.SIFTMatching(0, v3dm_mod.KERNEL_TCGEN05) as m:
        m.allocate(3000, 3500)
        m.set_left_features(L)
        m.set_right_features(R)
        best, ms = m.autotune(0.7, 0.8, 2)
        assert 0 <= best < m.num_configs() and ms > 0
        assert m.config()[0] == best
        np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), oracle_mod.match(L, R, 0.7, 0.8))
