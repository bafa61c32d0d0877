"""Parity of the CUDA vocabulary-tree quantizer with the oracle and the reference quantizer."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bf,depth,n", [(2, 1, 10), (3, 2, 100), (4, 3, 1000), (10, 3, 5000), (10, 4, 20000),
                                        (50, 3, 3000), (300, 2, 2000), (7, 5, 333)])
def test_quantize_matches_oracle(v3dm_mod, oracle_mod, bf, depth, n):
    rng = synth.rng_for(bf * 100 + depth)
    nodes = synth.sift_like(rng, v3dm_mod.voctree_counts(bf, depth)[0])
    keys = synth.sift_like(rng, n)
    t = v3dm_mod.VocabularyTreeTraversal(bf, depth)
    t.allocate(n)
    t.set_nodes(nodes)
    for mode, glob in ((v3dm_mod.LEAF_GLOBAL, True), (v3dm_mod.LEAF_LOCAL, False)):
        got = t.traverse_tree(keys, mode)
        np.testing.assert_array_equal(got, oracle_mod.voctree(bf, depth, nodes, keys, glob))
    # float (u/512) inputs give the same ids
    t2 = v3dm_mod.VocabularyTreeTraversal(bf, depth)
    t2.allocate(n)
    t2.set_nodes(nodes.astype(np.float32) / 512)
    np.testing.assert_array_equal(t2.traverse_tree(keys.astype(np.float32) / 512), t.traverse_tree(keys))
    t.close()
    t2.close()


def test_ties_take_first_child(v3dm_mod, oracle_mod):
    bf, depth = 4, 2
    nodes = np.zeros((20, 128), np.uint8)
    nodes[:] = 10  # all children equal: every level takes child 0
    keys = synth.sift_like(synth.rng_for(1), 50)
    t = v3dm_mod.VocabularyTreeTraversal(bf, depth)
    t.allocate(50)
    t.set_nodes(nodes)
    got = t.traverse_tree(keys, v3dm_mod.LEAF_GLOBAL)
    assert np.all(got == 4)  # level-1 node 0 -> children (0+1)*4 + 0
    np.testing.assert_array_equal(got, oracle_mod.voctree(bf, depth, nodes, keys, True))


def test_hkm_tree_bf10_depth6(v3dm_mod, oracle_mod):
    """The 10^6-leaf tree shape with HKM centres, 200k queries."""
    rng = synth.rng_for(3)
    train = synth.sift_like(rng, 60000)
    nodes = synth.hkm_tree(rng, train, 10, 6, iters=2)
    keys = synth.sift_like(rng, 200000)
    t = v3dm_mod.VocabularyTreeTraversal(10, 6)
    t.allocate(keys.shape[0])
    t.set_nodes(nodes)
    got = t.traverse_tree(keys, v3dm_mod.LEAF_LOCAL)
    np.testing.assert_array_equal(got, oracle_mod.voctree(10, 6, nodes, keys, False))
