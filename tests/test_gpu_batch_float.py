"""Batched matching of float descriptors (v3dm_batch_set_images_f32).

The reference uploads float descriptors per image and matches pairs one at a time
(V3D/CUDA/v3d_cudamatching.cu:490-552; the loop of V3D/Apps/SfM/match_sequence.cpp:165-234).
Every pair's result of the batch equals, bit for bit, SIFTMatching's float findPutativeMatches
on the two images (the BF16 hi/lo scores of v3dm_match_f.cu and the reference's rules on them),
and every guided result that putative call followed by one runGuidedMatching /
runGuidedHomographyMatching with the pair's gate (.cu:554-694); images whose values are all u/512
take the integer layout, whose results equal the oracle's."""
import ctypes as C

import numpy as np
import pytest

from v3dm import synth
from float_util import float_images

pytestmark = pytest.mark.gpu


def _single(v3dm_mod, L, R, ms, mr):
    if L.shape[0] == 0 or R.shape[0] == 0:
        return np.zeros((0, 2), np.int32)
    with v3dm_mod.SIFTMatching(0) as m:
        m.allocate(L.shape[0], R.shape[0], False)
        m.set_left_features(L)
        m.set_right_features(R)
        return m.find_putative_matches(ms, mr)


def _single_guided(v3dm_mod, desc, pos, offs, i, j, homography, M, thr, ms, mr):
    L, R = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
    lp, rp = pos[offs[i]:offs[i + 1]], pos[offs[j]:offs[j + 1]]
    if L.shape[0] == 0 or R.shape[0] == 0:
        return np.zeros((0, 2), np.int32)
    with v3dm_mod.SIFTMatching(0) as m:
        m.allocate(L.shape[0], R.shape[0], True)
        m.set_left_features(L)
        m.set_right_features(R)
        m.find_putative_matches(ms, mr)
        if homography:
            return m.run_guided_homography_matching(M, float(thr), lp, rp, ms, mr)
        return m.run_guided_matching(M, float(thr), lp, rp, ms, mr)


def _ragged(desc, counts, offs, keep):
    parts, new = [], []
    for i, k in enumerate(keep):
        n = int(counts[i]) if k is None else min(k, int(counts[i]))
        parts.append(desc[offs[i]:offs[i] + n])
        new.append(n)
    counts = np.asarray(new, np.int32)
    return np.concatenate(parts), counts, np.concatenate([[0], np.cumsum(counts)])


@pytest.fixture(scope="module")
def ragged_float():
    """Eight float images: empty, one descriptor, sizes around the 128-row groups and the 64-column
    tiles, and image 6 kept at u/512 (mixed pairs)."""
    desc, counts, offs = float_images(31, 8, 300, 2600, exact=(6,))
    return _ragged(desc, counts, offs, [0, 1, 63, 129, 700, None, None, 1500])


def test_float_all_pairs_equal_single_pair_matcher(v3dm_mod, ragged_float):
    desc, counts, offs = ragged_float
    pairs = synth.all_pairs(len(counts))
    total = 0
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        assert b.float_mode
        b.set_pairs(None)
        for ms, mr in ((0.7, 0.8), (0.85, 0.6), (0.7, -1.0)):
            per = b.split_pairs(b.match(ms, mr))
            for k, (i, j) in enumerate(pairs):
                L, R = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
                np.testing.assert_array_equal(per[k], _single(v3dm_mod, L, R, ms, mr),
                                              err_msg=f"pair {k} ({i}, {j}) ms={ms} mr={mr}")
                total += len(per[k])
    assert total > 500


def test_float_custom_table_and_repeat(v3dm_mod, ragged_float):
    """Reversed, repeated and self pairs in arbitrary order; a second call (graph replay) gives
    the same triples."""
    desc, counts, offs = ragged_float
    pairs = np.array([[5, 4], [4, 5], [7, 6], [6, 7], [5, 5], [3, 7], [5, 4], [0, 5], [1, 7]], np.int32)
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(pairs)
        t = b.match(0.75, 0.8)
        np.testing.assert_array_equal(t, b.match(0.75, 0.8))
        per = b.split_pairs(t)
    for k, (i, j) in enumerate(pairs):
        L, R = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
        np.testing.assert_array_equal(per[k], _single(v3dm_mod, L, R, 0.75, 0.8), err_msg=f"pair {k} ({i}, {j})")


def test_exact_float_images_take_the_integer_layout(v3dm_mod, oracle_mod):
    desc, counts, offs = synth.images(32, 5, 200, 1200)
    f = desc.astype(np.float32) / 512
    pairs = synth.all_pairs(len(counts))
    with v3dm_mod.BatchMatching() as b:
        b.set_images(f, counts)
        assert not b.float_mode
        b.set_pairs(None)
        per = b.split_pairs(b.match(0.7, 0.8))
    for k, (i, j) in enumerate(pairs):
        exp = oracle_mod.match(desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]], 0.7, 0.8)
        np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k}")


def test_mode_switches_and_errors(v3dm_mod, oracle_mod):
    """Float -> uint8 -> float uploads of the same sizes (the graph of the other mode is
    dropped); guided and proposal calls need the integer layout; non-finite values and
    misaligned device pointers are argument errors."""
    import torch
    desc, counts, offs = float_images(33, 4, 300, 900)
    u8, _, _ = synth.images(33, 4, 300, 900)
    pairs = synth.all_pairs(4)
    L = v3dm_mod.lib()
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(None)
        first = b.match(0.7, 0.8)
        b.set_images(u8, counts)
        assert not b.float_mode
        per = b.split_pairs(b.match(0.7, 0.8))
        for k, (i, j) in enumerate(pairs):
            exp = oracle_mod.match(u8[offs[i]:offs[i + 1]], u8[offs[j]:offs[j + 1]], 0.7, 0.8)
            np.testing.assert_array_equal(per[k], exp)
        d = torch.from_numpy(desc).cuda()
        b.set_images_device(d.data_ptr(), counts, np.float32)
        assert b.float_mode
        np.testing.assert_array_equal(b.match(0.7, 0.8), first)
        # a guided call on float images needs positions
        F = np.zeros((b.n_pairs, 9))
        thr = np.ones(b.n_pairs, np.float32)
        out = np.empty((16, 3), np.int32)
        n = C.c_longlong(0)
        st = L.v3dm_batch_match_guided(b._h, 1, F.ctypes.data, thr.ctypes.data, 0.7, 0.8, out.ctypes.data, 16,
                                       C.byref(n))
        assert st == v3dm_mod.ERR_NOT_ALLOCATED
        # misaligned device pointer, non-finite value
        st = L.v3dm_batch_set_images_f32_device(b._h, 4, counts.ctypes.data, C.c_void_p(d.data_ptr() + 4))
        assert st == v3dm_mod.ERR_ARG
        bad = desc.copy()
        bad[5, 7] = np.nan
        with pytest.raises(Exception):
            b.set_images(bad, counts)
        # a good upload afterwards works again
        b.set_images(desc, counts)
        b.set_pairs(None)
        np.testing.assert_array_equal(b.match(0.7, 0.8), first)


def test_float_guided_equals_single_pair_guided(v3dm_mod):
    """Guided calls on float images (cameras along a line, tracks at their projections): every
    pair, F gates of 2 and 8 px and two parameter sets, then homography gates on a custom table,
    against the single-pair float matcher's putative call followed by one guided call."""
    desc8, counts, offs, pos, cams = synth.scene(23, 7, 300, 2600)
    desc = synth.float_from_u8(desc8, 23)
    pairs = synth.all_pairs(len(counts))
    F = np.stack([synth.fundamental(cams, i, j) for i, j in pairs])
    thr = np.where(np.arange(len(pairs)) % 3 == 0, 8.0, 2.0).astype(np.float32)
    total_g = total_p = 0
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        assert b.float_mode
        b.set_pairs(None)
        b.set_positions(pos)
        for ms, mr in ((0.7, 0.8), (0.6, 0.95)):
            per = b.split_pairs(b.match_guided(F, thr, ms, mr))
            put = b.split_pairs(b.match(ms, mr))
            for k, (i, j) in enumerate(pairs):
                exp = _single_guided(v3dm_mod, desc, pos, offs, i, j, False, F[k], thr[k], ms, mr)
                np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k} ({i}, {j}) ms={ms} mr={mr}")
                total_g += len(per[k])
                total_p += len(put[k])
        assert total_g > 100 and total_g != total_p  # the gates matter
        rng = np.random.default_rng(6)
        tab = np.array([[3, 5], [5, 3], [6, 2], [3, 5], [4, 4], [0, 6]], np.int32)
        H = np.stack([np.eye(3) + np.array([[rng.normal(0, 0.02), rng.normal(0, 0.02), rng.normal(0, 30)],
                                            [rng.normal(0, 0.02), rng.normal(0, 0.02), rng.normal(0, 30)],
                                            [rng.normal(0, 1e-5), rng.normal(0, 1e-5), 0.0]]) for _ in tab])
        th = rng.uniform(40.0, 400.0, len(tab)).astype(np.float32)
        b.set_pairs(tab)
        perH = b.split_pairs(b.match_guided(H, th, 0.6, 0.9, homography=True))
    n = 0
    for k, (i, j) in enumerate(tab):
        exp = _single_guided(v3dm_mod, desc, pos, offs, i, j, True, H[k], th[k], 0.6, 0.9)
        np.testing.assert_array_equal(perH[k], exp, err_msg=f"H pair {k} ({i}, {j})")
        n += len(exp)
    assert n > 0


def test_float_batch_at_scale_sampled(v3dm_mod):
    """24 float images of 1000..6000 descriptors, all 276 pairs: 10 sampled pairs against the
    single-pair float matcher, and the whole call against a second run."""
    desc, counts, offs = float_images(34, 24, 1000, 6000)
    pairs = synth.all_pairs(len(counts))
    with v3dm_mod.BatchMatching() as b:
        b.set_images(desc, counts)
        b.set_pairs(None)
        t = b.match(0.7, 0.8)
        np.testing.assert_array_equal(t, b.match(0.7, 0.8))
        per = b.split_pairs(t)
        launches = b.last_launches()
    assert launches == 7
    rng = np.random.default_rng(1)
    for k in rng.choice(len(pairs), 10, replace=False):
        i, j = pairs[k]
        L, R = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
        np.testing.assert_array_equal(per[k], _single(v3dm_mod, L, R, 0.7, 0.8), err_msg=f"pair {k} ({i}, {j})")
    assert t.shape[0] > 2000
