"""Retrieval scoring, CPU part: the oracle's restatement of the voctree app's image loop over
LeafDocuments (match_using_voctree.cpp:176-222; V3D/Base/v3d_voctree.h:143-278) against
fixtures written by the reference's own LeafDocuments and, when oracle/_ref is built, against
the reference live; and the library's pair-table conversion (v3dm_retrieval_pairs, host code)
against the app's map<int, set<int>> (match_using_voctree.cpp:196-216)."""
from pathlib import Path

import numpy as np
import pytest

from v3dm import synth

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden_cases():
    z = np.load(GOLDEN / "retrieval_ref.npz")
    for name in z["names"]:
        name = str(name)
        yield (name, int(z[f"{name}_n_leaves"]), z[f"{name}_offsets"], z[f"{name}_words"],
               float(z[f"{name}_p_match"]), z[f"{name}_docs"], z[f"{name}_scores"])


def _same(docs, sc, exp_docs, exp_sc):
    np.testing.assert_array_equal(docs, exp_docs)
    np.testing.assert_array_equal(sc.view(np.uint32), exp_sc.view(np.uint32))


def test_oracle_matches_reference_fixtures(oracle_mod):
    n = 0
    for name, n_leaves, off, w, pm, exp_docs, exp_sc in _golden_cases():
        for threads in (1, 0):
            docs, sc = oracle_mod.retrieval(n_leaves, off, w, pm, exp_docs.shape[1], threads)
            _same(docs, sc, exp_docs, exp_sc)
        n += 1
    assert n == 5


def test_fixture_edge_cases_are_present():
    """The edge fixture holds equal scores (identical images ranked by index), an empty image
    and a row shorter than n_best."""
    z = {c[0]: c for c in _golden_cases()}
    _, _, off, w, _, docs, sc = z["edges"]
    assert (np.diff(off) == 0).any()
    # images 3 and 4 are copies of image 0: image 4 sees 0 and 3 with one score, 0 first
    row = list(docs[4])
    assert row.index(0) < row.index(3) and sc[4, row.index(0)] == sc[4, row.index(3)]
    _, _, _, _, _, docs_all, _ = z["edges_all"]
    assert (docs_all[5, 5:] == -1).all() and (docs_all[5, :5] >= 0).all()
    assert (z["single"][5] == -1).all()


@pytest.mark.parametrize("n_images,n_leaves,n_best,p_match,zipf", [
    (1, 200, 1, 0.1, 1.1), (33, 300, 4, 0.1, 1.1), (65, 3000, 20, 0.05, 0.8), (140, 20000, 25, 0.2, 1.3),
])
def test_oracle_matches_reference_live(oracle_mod, n_images, n_leaves, n_best, p_match, zipf):
    if not oracle_mod.ref_retrieval_available():
        pytest.skip("reference LeafDocuments not built (oracle/_ref)")
    off, w = synth.sequence_words(n_images + n_leaves, n_images=n_images, n_leaves=n_leaves, n_min=10,
                                  n_max=max(10, min(400, n_leaves // 20)), window=5, zipf=zipf)
    exp = oracle_mod.ref_retrieval(n_leaves, off, w, p_match, n_best)
    _same(*oracle_mod.retrieval(n_leaves, off, w, p_match, n_best), *exp)


def test_oracle_rejects_words_out_of_range(oracle_mod):
    off = np.array([0, 2], np.int32)
    with pytest.raises(ValueError):
        oracle_mod.retrieval(5, off, np.array([1, 5], np.int32), 0.1, 2)


def _app_pairs(docs):
    """putativePairwiseMatches of match_using_voctree.cpp:196-216, listed as the .dot writer
    walks it (:224-233)."""
    m = {}
    for i in range(docs.shape[0]):
        for d in docs[i]:
            if d >= 0:
                m.setdefault(int(d), set()).add(i)
    return np.array([(v1, v2) for v1 in sorted(m) for v2 in sorted(m[v1])], np.int32).reshape(-1, 2)


def test_pair_table_matches_the_app(v3dm_mod, oracle_mod):
    for name, n_leaves, off, w, pm, docs, sc in _golden_cases():
        np.testing.assert_array_equal(v3dm_mod.retrieval_pairs(docs), _app_pairs(docs))
    off, w = synth.sequence_words(5, n_images=300, n_leaves=4000, n_min=50, n_max=150)
    docs, _ = oracle_mod.retrieval(4000, off, w, 0.1, 20)
    got = v3dm_mod.retrieval_pairs(docs)
    np.testing.assert_array_equal(got, _app_pairs(docs))
    assert (got[:, 0] < got[:, 1]).all() and got.shape[0] == sum(min(i, 20) for i in range(300))


def test_pair_table_errors(v3dm_mod):
    import ctypes as C
    L = v3dm_mod.lib()
    docs = np.array([[-1, -1], [0, -1], [1, 0]], np.int32)
    n = C.c_longlong(-1)
    assert L.v3dm_retrieval_pairs(3, 2, docs.ctypes.data, 0, None, C.byref(n)) == v3dm_mod.OK and n.value == 3
    out = np.full((3, 2), -7, np.int32)
    assert L.v3dm_retrieval_pairs(3, 2, docs.ctypes.data, 2, out.ctypes.data, C.byref(n)) == v3dm_mod.ERR_CAPACITY
    np.testing.assert_array_equal(out[:2], [[0, 1], [0, 2]])
    assert (out[2] == -7).all()
    bad = np.array([[-1], [1]], np.int32)  # image 1 cannot retrieve itself
    assert L.v3dm_retrieval_pairs(2, 1, bad.ctypes.data, 0, None, C.byref(n)) == v3dm_mod.ERR_ARG
    assert L.v3dm_retrieval_pairs(2, 0, docs.ctypes.data, 0, None, C.byref(n)) == v3dm_mod.ERR_ARG


@pytest.mark.parametrize("p_match,n_best,n_min,n_max", [(0.0, 3, 1, 30), (0.3, 60, 1, 20), (0.1, 1, 1, 1),
                                                        (0.05, 7, 100, 400)])
def test_oracle_matches_reference_varied(oracle_mod, p_match, n_best, n_min, n_max):
    """pMatch 0 and 0.3, nBest above the image count, images of a single word."""
    if not oracle_mod.ref_retrieval_available():
        pytest.skip("reference LeafDocuments not built (oracle/_ref)")
    off, w = synth.sequence_words(int(p_match * 100) + n_best, n_images=45, n_leaves=2000, n_min=n_min, n_max=n_max,
                                  window=4, zipf=0.9)
    exp = oracle_mod.ref_retrieval(2000, off, w, p_match, n_best)
    _same(*oracle_mod.retrieval(2000, off, w, p_match, n_best), *exp)
