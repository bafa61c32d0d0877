"""Retrieval scoring on the GPU (v3dm_retrieval_*): bit-exact against the fixtures written by
the reference's LeafDocuments (V3D/Base/v3d_voctree.h:143-278 in the loop of
match_using_voctree.cpp:176-222) and against the oracle's restatement (pinned to the same
fixtures by tests/test_retrieval.py) on sequences up to the bench's size; the device-resident
call; errors; the LeafDocuments mirror; and the pair table feeding the batched matcher."""
from pathlib import Path

import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _same(docs, sc, exp_docs, exp_sc):
    np.testing.assert_array_equal(docs, exp_docs)
    np.testing.assert_array_equal(sc.view(np.uint32), exp_sc.view(np.uint32))


def test_golden_fixtures(v3dm_mod):
    z = np.load(GOLDEN / "retrieval_ref.npz")
    with v3dm_mod.Retrieval() as r:
        for name in z["names"]:
            name = str(name)
            exp_docs, exp_sc = z[f"{name}_docs"], z[f"{name}_scores"]
            got = r.binomial(int(z[f"{name}_n_leaves"]), z[f"{name}_offsets"], z[f"{name}_words"],
                             float(z[f"{name}_p_match"]), exp_docs.shape[1])
            _same(*got, exp_docs, exp_sc)


@pytest.mark.parametrize("n_images,n_leaves,n_min,n_max,n_best,p_match,zipf", [
    (2, 100, 0, 5, 1, 0.1, 1.1),
    (32, 500, 1, 40, 3, 0.1, 1.1),
    (33, 500, 1, 40, 40, 0.0, 1.1),
    (257, 20000, 50, 400, 20, 0.1, 1.2),
    (700, 125000, 500, 2500, 20, 0.1, 1.1),
    (1100, 60000, 100, 900, 300, 0.05, 1.3),
    (2048, 125000, 2000, 6000, 20, 0.1, 1.1),
])
def test_matches_oracle(v3dm_mod, oracle_mod, n_images, n_leaves, n_min, n_max, n_best, p_match, zipf):
    off, w = synth.sequence_words(n_images * 7 + n_best, n_images=n_images, n_leaves=n_leaves, n_min=n_min,
                                  n_max=n_max, window=6, zipf=zipf)
    if n_min == 0:  # at most one empty image (two empty images score NaN)
        cnt = np.diff(off)
        assert (cnt == 0).sum() <= 1
    exp = oracle_mod.retrieval(n_leaves, off, w, p_match, n_best)
    with v3dm_mod.Retrieval() as r:
        _same(*r.binomial(n_leaves, off, w, p_match, n_best), *exp)
        # a second call on the same object (buffers reused) and a smaller one after it
        _same(*r.binomial(n_leaves, off, w, p_match, n_best), *exp)
        k = max(1, n_images // 3)
        _same(*r.binomial(n_leaves, off[:k + 1], w[:off[k]], p_match, n_best),
              *oracle_mod.retrieval(n_leaves, off[:k + 1], w[:off[k]], p_match, n_best))


def test_huge_images_and_long_sequences(v3dm_mod, oracle_mod):
    """Images with more rows than one counter segment (32752) and one staged chunk (4096), and a
    sequence long enough (> 16384 images) that a query reads its bitmap columns in two passes."""
    off, w = synth.sequence_words(31, n_images=24, n_leaves=400_000, n_min=20_000, n_max=70_000)
    exp = oracle_mod.retrieval(400_000, off, w, 0.1, 6)
    with v3dm_mod.Retrieval() as r:
        _same(*r.binomial(400_000, off, w, 0.1, 6), *exp)
    off, w = synth.sequence_words(32, n_images=16_500, n_leaves=3000, n_min=1, n_max=12, window=3)
    exp = oracle_mod.retrieval(3000, off, w, 0.1, 5)
    with v3dm_mod.Retrieval() as r:
        _same(*r.binomial(3000, off, w, 0.1, 5), *exp)


def test_max_best_and_many_images(v3dm_mod, oracle_mod):
    off, w = synth.sequence_words(21, n_images=1500, n_leaves=30000, n_min=20, n_max=200)
    nb = v3dm_mod.RETRIEVAL_MAX_BEST
    exp = oracle_mod.retrieval(30000, off, w, 0.1, nb)
    with v3dm_mod.Retrieval() as r:
        _same(*r.binomial(30000, off, w, 0.1, nb), *exp)


def test_device_call_and_pair_table(v3dm_mod, oracle_mod):
    import torch
    off, w = synth.sequence_words(8, n_images=400, n_leaves=50000, n_min=300, n_max=1200)
    nb = 10
    exp_docs, exp_sc = oracle_mod.retrieval(50000, off, w, 0.1, nb)
    dw = torch.from_numpy(w).cuda()
    docs = torch.empty((400, nb), dtype=torch.int32, device="cuda")
    sc = torch.empty((400, nb), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    with v3dm_mod.Retrieval() as r:
        r.binomial_device(50000, off, dw.data_ptr(), 0.1, nb, docs.data_ptr(), sc.data_ptr())
        r.wait()
        _same(docs.cpu().numpy(), sc.cpu().numpy(), exp_docs, exp_sc)
        # a word out of range is reported by wait (and skipped)
        bad = w.copy()
        bad[5] = 50000
        dbad = torch.from_numpy(bad).cuda()
        torch.cuda.synchronize()
        r.binomial_device(50000, off, dbad.data_ptr(), 0.1, nb, docs.data_ptr(), sc.data_ptr())
        with pytest.raises(v3dm_mod.V3DMError) as e:
            r.wait()
        assert e.value.status == v3dm_mod.ERR_ARG
        r.wait()  # the error was consumed
    pairs = v3dm_mod.retrieval_pairs(exp_docs)
    assert pairs.shape[0] == sum(min(i, nb) for i in range(400))
    # the retrieved pairs feed the batched matcher as its pair table
    desc, counts, offs = synth.images(17, n_images=12, n_min=500, n_max=1500)
    off12, w12 = synth.sequence_words(9, n_images=12, n_leaves=5000, n_min=200, n_max=400)
    with v3dm_mod.Retrieval() as r:
        d12, _ = r.binomial(5000, off12, w12, 0.1, 3)
    p12 = v3dm_mod.retrieval_pairs(d12)
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(p12)
    per = b.match_per_pair(0.7, 0.8)
    b.close()
    assert len(per) == p12.shape[0] and sum(len(x) for x in per) > 0
    m = v3dm_mod.SIFTMatching()
    m.allocate(1500, 1500)
    for k, (a, c) in enumerate(p12):
        m.set_left_features(desc[offs[a]:offs[a + 1]])
        m.set_right_features(desc[offs[c]:offs[c + 1]])
        np.testing.assert_array_equal(per[k], m.find_putative_matches(0.7, 0.8), err_msg=f"pair {k}")
    m.close()


def test_errors(v3dm_mod):
    import ctypes as C
    L = v3dm_mod.lib()
    off = np.array([0, 2, 4], np.int32)
    w = np.array([0, 1, 1, 7], np.int32)
    docs = np.empty((2, 2), np.int32)
    sc = np.empty((2, 2), np.float32)
    with v3dm_mod.Retrieval() as r:
        h = r._h
        args = lambda nl, n, o, nb: (h, nl, n, o.ctypes.data, w.ctypes.data, C.c_double(0.1), nb, docs.ctypes.data,
                                     sc.ctypes.data)
        assert L.v3dm_retrieval_binomial(*args(8, 2, off, 2)) == v3dm_mod.OK
        assert L.v3dm_retrieval_binomial(*args(7, 2, off, 2)) == v3dm_mod.ERR_ARG      # word 7 >= 7 leaves
        assert L.v3dm_retrieval_binomial(*args(8, 2, off, 0)) == v3dm_mod.ERR_ARG      # n_best 0
        assert L.v3dm_retrieval_binomial(*args(8, 2, off, v3dm_mod.RETRIEVAL_MAX_BEST + 1)) == v3dm_mod.ERR_ARG
        assert L.v3dm_retrieval_binomial(*args(8, 2, np.array([0, 3, 2], np.int32), 2)) == v3dm_mod.ERR_ARG
        assert L.v3dm_retrieval_binomial(*args(8, 2, np.array([1, 2, 4], np.int32), 2)) == v3dm_mod.ERR_ARG
        big = np.zeros(v3dm_mod.RETRIEVAL_MAX_IMAGES + 2, np.int32)
        assert L.v3dm_retrieval_binomial(*args(8, v3dm_mod.RETRIEVAL_MAX_IMAGES + 1, big, 2)) == v3dm_mod.ERR_SIZE
        assert L.v3dm_retrieval_binomial(*args(8, 0, off, 2)) == v3dm_mod.OK           # nothing to do
        # still usable
        d, s = r.binomial(8, off, w, 0.1, 2)
        assert d[1, 0] == 0 and d[0, 0] == -1


def test_leaf_documents_mirror(v3dm_mod, oracle_mod):
    """Code written against LeafDocuments' incremental interface gets the loop's scores."""
    off, w = synth.sequence_words(3, n_images=40, n_leaves=3000, n_min=50, n_max=200)
    exp_docs, exp_sc = oracle_mod.retrieval(3000, off, w, 0.1, 5)
    inv = v3dm_mod.LeafDocuments(3000)
    for i in range(40):
        q = w[off[i]:off[i + 1]]
        scores = inv.compute_binomial_scores(0.1, q, 5)
        assert [d for _, d in scores] == list(exp_docs[i, :min(i, 5)])
        assert np.array([s for s, _ in scores], np.float32).tobytes() == exp_sc[i, :min(i, 5)].tobytes()
        assert inv.insert_document(q) == i
    full = inv.compute_binomial_scores(0.1, w[off[7]:off[8]])  # every document, sorted
    assert len(full) == 40 and [s for s, _ in full] == sorted(s for s, _ in full)
