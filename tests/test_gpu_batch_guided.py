"""Batched guided matching (v3dm_batch_match_guided): every pair's result equals the oracle's
runGuidedMatching / runGuidedHomographyMatching with that pair's gate after its
findPutativeMatches (V3D/CUDA/v3d_cudamatching.cu:554-694), bit for bit -- the apps' per-pair
sequence putative -> RANSAC -> guided (V3D/Apps/SfM/match_sequence.cpp:306-324) for a batch."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    """Cameras along a line, shared tracks at their projections (1 px noise), sizes that cover
    empty, tiny and ragged images."""
    desc, counts, offs, pos, cams = synth.scene(21, 9, 300, 2600)
    counts = counts.copy()
    # ragged sizes: drop features from some images (keep the geometry of the rest)
    keep = [0, 40, 257, None, 1, None, 700, None, 1023]
    parts_d, parts_p, new_counts = [], [], []
    for i, k in enumerate(keep):
        n = int(counts[i]) if k is None else min(k, int(counts[i]))
        parts_d.append(desc[offs[i]:offs[i] + n])
        parts_p.append(pos[offs[i]:offs[i] + n])
        new_counts.append(n)
    desc = np.concatenate(parts_d)
    pos = np.concatenate(parts_p)
    counts = np.asarray(new_counts, np.int32)
    offs = np.concatenate([[0], np.cumsum(counts)])
    return desc, counts, offs, pos, cams


def _oracle_pair(oracle_mod, desc, pos, offs, i, j, kind, M, thr, ms, mr):
    L, R = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
    lp, rp = pos[offs[i]:offs[i + 1]], pos[offs[j]:offs[j + 1]]
    return oracle_mod.match(L, R, ms, mr, gates=[(kind, M, float(thr))], lpos=lp, rpos=rp)


def test_guided_all_pairs_equal_oracle(v3dm_mod, oracle_mod, scene):
    desc, counts, offs, pos, cams = scene
    pairs = synth.all_pairs(len(counts))
    F = np.stack([synth.fundamental(cams, i, j) for i, j in pairs])
    thr = np.where(np.arange(len(pairs)) % 3 == 0, 8.0, 2.0).astype(np.float32)
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(None)
        b.set_positions(pos)
        total_guided = total_put = 0
        for ms, mr in ((0.7, 0.8), (0.6, 0.95), (0.7, -1.0)):
            per = b.split_pairs(b.match_guided(F, thr, ms, mr))
            put = b.match_per_pair(ms, mr)
            for k, (i, j) in enumerate(pairs):
                exp = _oracle_pair(oracle_mod, desc, pos, offs, i, j, "F", F[k], thr[k], ms, mr)
                np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k} ({i}, {j}) ms={ms} mr={mr}")
                total_guided += len(per[k])
                total_put += len(put[k])
        # the gate matters: the guided results are not the putative ones
        assert total_guided > 100 and total_guided != total_put


def test_guided_homography_and_custom_table(v3dm_mod, oracle_mod, scene):
    """Homography gates, a pair table in arbitrary order with reversed, repeated and self pairs."""
    desc, counts, offs, pos, _ = scene
    rng = np.random.default_rng(5)
    pairs = np.array([[3, 5], [5, 3], [8, 2], [3, 5], [4, 4], [0, 6], [6, 0], [2, 8], [7, 3]], np.int32)
    H = np.stack([np.eye(3) + np.array([[rng.normal(0, 0.02), rng.normal(0, 0.02), rng.normal(0, 30)],
                                        [rng.normal(0, 0.02), rng.normal(0, 0.02), rng.normal(0, 30)],
                                        [rng.normal(0, 1e-5), rng.normal(0, 1e-5), 0.0]]) for _ in pairs])
    thr = rng.uniform(40.0, 400.0, len(pairs)).astype(np.float32)
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(pairs)
        b.set_positions(pos)
        per = b.split_pairs(b.match_guided(H, thr, 0.6, 0.9, homography=True))
    n = 0
    for k, (i, j) in enumerate(pairs):
        exp = _oracle_pair(oracle_mod, desc, pos, offs, i, j, "H", H[k], thr[k], 0.6, 0.9)
        np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k} ({i}, {j})")
        n += len(exp)
    assert n > 0


def test_guided_equals_single_pair_guided_call(v3dm_mod, scene):
    """Same result as SIFTMatching: putative call, then one guided call on the same pair."""
    desc, counts, offs, pos, cams = scene
    pairs = np.array([[3, 5], [7, 8], [5, 7]], np.int32)
    F = np.stack([synth.fundamental(cams, i, j) for i, j in pairs])
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(pairs)
        b.set_positions(pos)
        per = b.split_pairs(b.match_guided(F, 2.0, 0.7, 0.8))
    for k, (i, j) in enumerate(pairs):
        L, R = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
        with v3dm_mod.SIFTMatching(0) as m:
            m.allocate(L.shape[0], R.shape[0], True)
            m.set_left_features(L)
            m.set_right_features(R)
            m.find_putative_matches(0.7, 0.8)
            exp = m.run_guided_matching(F[k], 2.0, pos[offs[i]:offs[i + 1]], pos[offs[j]:offs[j + 1]], 0.7, 0.8)
        np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k}")


def test_guided_batch_at_scale_sampled(v3dm_mod, oracle_mod):
    """24 images of 1000..6000 features, all 276 pairs; 12 sampled pairs checked against the
    oracle, and the whole call against a second run (deterministic output)."""
    desc, counts, offs, pos, cams = synth.scene(22, 24, 1000, 6000)
    pairs = synth.all_pairs(len(counts))
    F = np.stack([synth.fundamental(cams, i, j) for i, j in pairs])
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(None)
        b.set_positions(pos)
        t = b.match_guided(F, 2.0, 0.7, 0.8)
        np.testing.assert_array_equal(t, b.match_guided(F, 2.0, 0.7, 0.8))
        per = b.split_pairs(t)
    rng = np.random.default_rng(0)
    for k in rng.choice(len(pairs), 12, replace=False):
        i, j = pairs[k]
        exp = _oracle_pair(oracle_mod, desc, pos, offs, i, j, "F", F[k], 2.0, 0.7, 0.8)
        np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k} ({i}, {j})")
    assert t.shape[0] > 1000


def test_guided_argument_errors(v3dm_mod, scene):
    import ctypes as C
    desc, counts, offs, pos, cams = scene
    L = v3dm_mod.lib()
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(None)
        F = np.zeros((b.n_pairs, 9))
        thr = np.ones(b.n_pairs, np.float32)
        out = np.empty((16, 3), np.int32)
        n = C.c_longlong(0)
        # no positions yet
        st = L.v3dm_batch_match_guided(b._h, 1, F.ctypes.data, thr.ctypes.data, 0.7, 0.8, out.ctypes.data, 16,
                                       C.byref(n))
        assert st == v3dm_mod.ERR_NOT_ALLOCATED
        b.set_positions(pos)
        for typ in (0, 3):
            st = L.v3dm_batch_match_guided(b._h, typ, F.ctypes.data, thr.ctypes.data, 0.7, 0.8, out.ctypes.data, 16,
                                           C.byref(n))
            assert st == v3dm_mod.ERR_ARG
        st = L.v3dm_batch_match_guided(b._h, 1, None, thr.ctypes.data, 0.7, 0.8, out.ctypes.data, 16, C.byref(n))
        assert st == v3dm_mod.ERR_ARG
        # new images drop the positions
        b.set_images(desc, counts)
        st = L.v3dm_batch_match_guided(b._h, 1, F.ctypes.data, thr.ctypes.data, 0.7, 0.8, out.ctypes.data, 16,
                                       C.byref(n))
        assert st == v3dm_mod.ERR_NOT_ALLOCATED
