"""Batched matching of many image pairs (v3dm_batch_*): every pair's result equals the oracle's
findPutativeMatches on the two images (V3D/CUDA/v3d_cudamatching.cu:522-552), bit for bit."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


def _images(seed, counts, track_frac=0.15):
    """Images with the given counts and shared tracks (noisy copies of common descriptors)."""
    rng = synth.rng_for(seed)
    counts = np.asarray(counts, np.int64)
    n_tracks = max(1, int(track_frac * counts.sum() / 4))
    base = synth.sift_like(rng, n_tracks)
    parts = []
    for c in counts:
        k = int(round(track_frac * c))
        k = min(k, c)
        tr = rng.integers(0, n_tracks, k)
        feats = np.concatenate([synth.noisy_copy(rng, base[tr]), synth.sift_like(rng, int(c) - k)])
        parts.append(feats[rng.permutation(int(c))])
    desc = np.concatenate(parts) if parts else np.zeros((0, 128), np.uint8)
    offs = np.concatenate([[0], np.cumsum(counts)])
    return desc, counts.astype(np.int32), offs


def _img(desc, offs, i):
    return desc[offs[i]:offs[i + 1]]


def _check_against_oracle(oracle_mod, desc, offs, pairs, per_pair, ms, mr):
    for k, (i, j) in enumerate(pairs):
        exp = oracle_mod.match(_img(desc, offs, i), _img(desc, offs, j), ms, mr)
        np.testing.assert_array_equal(per_pair[k], exp, err_msg=f"pair {k} ({i}, {j}) ms={ms} mr={mr}")


@pytest.fixture(scope="module")
def small_set():
    counts = [1500, 0, 1, 33, 2500, 700, 1024, 255, 257, 1999, 64, 1200, 3000, 900]
    return _images(11, counts)


def test_all_pairs_equal_oracle(v3dm_mod, oracle_mod, small_set):
    desc, counts, offs = small_set
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    pairs = synth.all_pairs(len(counts))
    assert b.n_pairs == len(pairs)
    for ms, mr in ((0.7, 0.8), (0.9, 0.8), (0.7, -1.0), (0.6, 0.95)):
        per = b.match_per_pair(ms, mr)
        _check_against_oracle(oracle_mod, desc, offs, pairs, per, ms, mr)
    assert sum(len(p) for p in b.match_per_pair(0.7, 0.8)) > 100
    b.close()


def test_custom_pair_table(v3dm_mod, oracle_mod, small_set):
    """Arbitrary order, repeated pairs, reversed pairs, self pairs, pairs with empty images."""
    desc, counts, offs = small_set
    pairs = np.array([[4, 0], [0, 4], [12, 12], [1, 5], [5, 1], [2, 3], [4, 0], [13, 6], [6, 13], [9, 8], [3, 2]],
                     np.int32)
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(pairs)
    per = b.match_per_pair(0.7, 0.8)
    _check_against_oracle(oracle_mod, desc, offs, pairs, per, 0.7, 0.8)
    # size-independent properties: the mutual filter is symmetric, repeats are identical
    np.testing.assert_array_equal(per[0], per[6])
    np.testing.assert_array_equal(per[1], per[0][:, ::-1][np.argsort(per[0][:, 1], kind="stable")])
    np.testing.assert_array_equal(per[8], per[7][:, ::-1][np.argsort(per[7][:, 1], kind="stable")])
    # an image matched with itself: descriptors match themselves (except repeated track views)
    assert len(per[2]) > 0.95 * counts[12] and np.all(per[2][:, 0] == per[2][:, 1])
    b.close()


def test_graph_replay_and_parameters(v3dm_mod, small_set):
    desc, counts, _ = small_set
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    a1 = b.match(0.7, 0.8)
    a2 = b.match(0.7, 0.8)  # graph replay
    c1 = b.match(0.9, 0.7)  # new parameters: new graph
    b.use_graph(False)
    a3 = b.match(0.7, 0.8)
    c2 = b.match(0.9, 0.7)
    np.testing.assert_array_equal(a1, a2)
    np.testing.assert_array_equal(a1, a3)
    np.testing.assert_array_equal(c1, c2)
    assert len(c1) < len(a1)
    b.close()


def test_every_config_and_schedule(v3dm_mod, small_set):
    desc, counts, _ = small_set
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    ref = None
    n_cfg = v3dm_mod.SIFTMatching().num_configs()
    for cfg in range(n_cfg):
        for sch in (0, 1, 2):
            b.set_config(cfg, sch)
            got = b.match(0.7, 0.8)
            if ref is None:
                ref = got
            np.testing.assert_array_equal(got, ref, err_msg=f"cfg {cfg} schedule {sch}")
    c, s, ms = b.autotune(0.7, 0.8, 1)
    assert b.config() == (c, s) and ms.shape == (n_cfg, 2) and np.all(ms > 0)
    np.testing.assert_array_equal(b.match(0.7, 0.8), ref)
    b.close()


def test_device_call_and_growth(v3dm_mod, oracle_mod):
    """Identical images: every left is accepted in every pair, far beyond the first pass-B
    buffers, so the call overflows once, grows them and is repeated."""
    rng = synth.rng_for(5)
    one = synth.sift_like(rng, 3000)
    n_img = 12
    desc = np.concatenate([one] * n_img)
    counts = np.full(n_img, 3000, np.int32)
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    t = b.match(0.7, 0.8)
    exp = oracle_mod.match(one, one, 0.7, 0.8)
    assert len(exp) > 2900
    assert len(t) == len(exp) * n_img * (n_img - 1) // 2
    per = b.match_per_pair(0.7, 0.8)
    for p in per:
        np.testing.assert_array_equal(p, exp)
    import torch
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    b.match_device(0.7, 0.8, cnt.data_ptr())
    assert b.wait() == v3dm_mod.OK
    assert int(cnt.item()) == len(t)
    b.close()


def test_config2_all_pairs_full_size(v3dm_mod, oracle_mod):
    """200 images with 1000..12000 features and shared tracks, all 19,900 pairs: a sample of
    pairs against the single-pair matcher and the oracle, and the symmetry of the mutual filter
    over the whole table."""
    desc, counts, offs = synth.images(2)
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    per = b.match_per_pair(0.7, 0.8)
    pairs = synth.all_pairs(len(counts))
    assert len(per) == 19900
    total = sum(len(p) for p in per)
    assert total > 10000
    rng = np.random.default_rng(0)
    sample = rng.choice(len(pairs), 40, replace=False)
    m = v3dm_mod.SIFTMatching()
    m.allocate(12000, 12000)
    for k in sample:
        i, j = pairs[k]
        m.set_left_features(_img(desc, offs, i))
        m.set_right_features(_img(desc, offs, j))
        np.testing.assert_array_equal(per[k], m.find_putative_matches(0.7, 0.8), err_msg=f"pair {k}")
    m.close()
    for k in sample[:4]:
        i, j = pairs[k]
        np.testing.assert_array_equal(per[k], oracle_mod.match(_img(desc, offs, i), _img(desc, offs, j), 0.7, 0.8))
    # reversed table: every pair's result is the transpose of the forward one
    b.set_pairs(pairs[:, ::-1].copy())
    rev = b.match_per_pair(0.7, 0.8)
    for k in range(0, len(pairs), 97):
        fwd = per[k][:, ::-1]
        np.testing.assert_array_equal(rev[k], fwd[np.argsort(fwd[:, 0], kind="stable")])
    b.close()
