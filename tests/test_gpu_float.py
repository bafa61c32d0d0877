"""Float descriptors through the BF16 hi/lo path (v3dm_match_f.cu), tcgen05 handle.

- u/512 descriptors through that path give the integer path's scores and pairs exactly;
- on arbitrary float descriptors the scores' error against float64 is bounded (stated in the
  test: 2e-5 absolute for unit-length descriptors) and the pairs are exactly the reference
  rules applied to the path's own scores (the selection with the float candidate threshold
  loses nothing);
- against the reference's own CUDA matcher (FP32 cublasSgemm, fast math) the pairs agree up
  to the few whose decision sits within the score error of a threshold."""
import numpy as np
import pytest

from v3dm import synth
from float_util import float_descriptors, reference_pairs

pytestmark = pytest.mark.gpu


@pytest.fixture
def matcher(v3dm_mod):
    made = []

    def make(nL, nR, guided=False):
        m = v3dm_mod.SIFTMatching(0, v3dm_mod.KERNEL_TCGEN05)
        m.allocate(nL, nR, guided)
        made.append(m)
        return m

    yield make
    for m in made:
        m.close()


@pytest.mark.parametrize("nL,nR", [(2000, 2100), (300, 1000), (1, 64), (129, 65)])
def test_u8_through_float_path_is_exact(matcher, oracle_mod, nL, nR):
    L, R, _ = synth.pair(nL + nR, nL, nR)
    m = matcher(nL, nR)
    m.set_left_features_bf16x3(L.astype(np.float32) / 512)
    m.set_right_features_bf16x3(R.astype(np.float32) / 512)
    S = m.scores_f32()
    exact = (L.astype(np.int64) @ R.astype(np.int64).T).astype(np.float32) * np.float32(2.0 ** -18)
    np.testing.assert_array_equal(S, exact)
    for ms, mr in ((0.7, 0.8), (0.9, 0.8), (0.7, -1.0)):
        np.testing.assert_array_equal(m.find_putative_matches(ms, mr), oracle_mod.match(L, R, ms, mr))
    # one side float, the other uint8 (built from the uint8 values, exactly)
    m.set_right_features(R)
    np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), oracle_mod.match(L, R, 0.7, 0.8))


def test_u8_guided_through_float_path_is_exact(matcher, oracle_mod):
    L, R, lp, rp, F, _ = synth.stereo(4, 2000, 2100)
    m = matcher(2000, 2100, True)
    m.set_left_features_bf16x3(L.astype(np.float32) / 512)
    m.set_right_features_bf16x3(R.astype(np.float32) / 512)
    np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), oracle_mod.match(L, R, 0.7, 0.8))
    got = m.run_guided_matching(F, 2.0, lp, rp, 0.7, 0.8)
    exp = oracle_mod.match(L, R, 0.7, 0.8, gates=[("F", F, 2.0)], lpos=lp, rpos=rp)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("seed,nL,nR", [(0, 3000, 2900), (1, 1500, 4000)])
def test_float_scores_error_and_selection(matcher, seed, nL, nR):
    L, R = float_descriptors(seed, nL, nR)
    m = matcher(nL, nR)
    m.set_left_features(L)  # not u/512: the float path
    m.set_right_features(R)
    S = m.scores_f32()
    S64 = L.astype(np.float64) @ R.astype(np.float64).T
    err = np.abs(S.astype(np.float64) - S64).max()
    assert err <= 2e-5, err
    for ms, mr in ((0.7, 0.8), (0.8, 0.6), (0.7, -1.0)):
        got = m.find_putative_matches(ms, mr)
        np.testing.assert_array_equal(got, reference_pairs(S, ms, mr))
        assert got.shape[0] > 50


def test_float_guided_selection(matcher):
    """Guided F on float descriptors: the reference's gate and rules on the path's scores."""
    import pyref
    L, R = float_descriptors(5, 320, 352)
    _, _, lp, rp, F, _ = synth.stereo(5, 320, 352)
    m = matcher(320, 352, True)
    m.set_left_features(L)
    m.set_right_features(R)
    S = m.scores_f32()
    put = m.find_putative_matches(0.7, 0.8)
    np.testing.assert_array_equal(put, reference_pairs(S, 0.7, 0.8))
    got = m.run_guided_matching(F, 40.0, lp, rp, 0.7, 0.8)
    masked = pyref.epipolar_mask(F, 40.0, lp, rp, S.T.copy())
    exp = pyref.match_from_scores(masked, 0.7, 0.8)[0]
    np.testing.assert_array_equal(got, exp)


def test_float_against_reference_gpu_matcher(matcher, oracle_mod, tmp_path):
    if not oracle_mod.ref_cuda_available():
        pytest.fail("oracle/_ref/libv3dref_cuda.so is missing")
    L, R = float_descriptors(7, 4096, 4096)
    m = matcher(4096, 4096)
    m.set_left_features(L)
    m.set_right_features(R)
    for ms, mr in ((0.7, 0.8), (0.8, 0.6)):
        got = {tuple(p) for p in m.find_putative_matches(ms, mr).tolist()}
        ref = {tuple(p) for p in oracle_mod.ref_cuda_match_f32(L, R, ms, mr, workdir=str(tmp_path)).tolist()}
        assert len(ref) > 100
        assert len(got ^ ref) <= max(2, len(ref) // 1000), (len(got), len(ref), len(got ^ ref))
