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


@pytest.mark.parametrize("bf,depth,n,vmax", [(2, 6, 5000, 3), (5, 4, 20000, 2), (11, 4, 30000, 255), (15, 2, 5000, 1),
                                             (10, 5, 200000, 4), (3, 1, 100, 255), (13, 3, 12000, 255)])
def test_tensor_descent_shapes_and_ties(v3dm_mod, oracle_mod, bf, depth, n, vmax):
    """Shapes the tensor-core descent takes (two levels per phase, 128-key tiles, the chosen
    child's grandchildren selected out of all BF^2 scores) with values drawn from 0..vmax: small
    vmax makes equal scores common, so the first-child rule is exercised at every level; 255 gives
    the largest scores."""
    rng = synth.rng_for(7000 + bf * 10 + depth)
    nodes = rng.integers(0, vmax + 1, (v3dm_mod.voctree_counts(bf, depth)[0], 128)).astype(np.uint8)
    keys = rng.integers(0, vmax + 1, (n, 128)).astype(np.uint8)
    keys[0] = 0  # a zero key ties everywhere
    keys[1] = vmax
    with v3dm_mod.VocabularyTreeTraversal(bf, depth) as t:
        t.allocate(n)
        t.set_nodes(nodes)
        for mode, glob in ((v3dm_mod.LEAF_GLOBAL, True), (v3dm_mod.LEAF_LOCAL, False)):
            np.testing.assert_array_equal(t.traverse_tree(keys, mode), oracle_mod.voctree(bf, depth, nodes, keys, glob))


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


def _ref_or_port(oracle_mod, bf, depth, nodes, keys):
    """Leaf-local ids of the reference's own CPU tree (VocabularyTree::getVisualWord, built from
    the reference headers into oracle/_ref) when that build is present, and the oracle's
    restatement of it; both must agree."""
    port = oracle_mod.voctree(bf, depth, nodes, keys, False)
    if oracle_mod.ref_voctree_available():
        ref = oracle_mod.ref_voctree(bf, depth, nodes, keys)
        np.testing.assert_array_equal(port, ref)
    return port


@pytest.mark.parametrize("bf,depth,n_train,n", [(10, 5, 60000, 100000), (50, 3, 40000, 60000),
                                                (300, 2, 40000, 40000), (10, 6, 150000, 200000)])
def test_float_tree_equals_reference_cpu_tree(v3dm_mod, oracle_mod, bf, depth, n_train, n):
    """Float k-means trees of unit-L2 descriptors (the apps' trees, v3d_voctree.h:38-52) and
    unit-L2 float keys: leaf ids equal the reference CPU tree's sequential FP32 descent, for the
    GPU class's instantiated shapes (.cu:866-868) and the 10^6-leaf tree, both id modes, host
    and device entry points."""
    import torch
    nodes, keys = synth.voctree(40 + bf, bf, depth, n_train, n, iters=2, floats=True)
    assert nodes.dtype == np.float32 and not np.array_equal(nodes * 512, np.rint(nodes * 512))
    keys[7] = np.nan  # the reference keeps child -1 at every level for a NaN key
    keys[8] = 0.0     # every score 0: ties, first child
    exp_local = _ref_or_port(oracle_mod, bf, depth, nodes, keys)
    leaf_base = v3dm_mod.voctree_counts(bf, depth)[0] - v3dm_mod.voctree_counts(bf, depth)[1]
    t = v3dm_mod.VocabularyTreeTraversal(bf, depth)
    t.allocate(n)
    t.set_nodes(nodes)
    np.testing.assert_array_equal(t.traverse_tree(keys, v3dm_mod.LEAF_LOCAL), exp_local)
    np.testing.assert_array_equal(t.traverse_tree(keys, v3dm_mod.LEAF_GLOBAL), exp_local + leaf_base)
    d_keys = torch.from_numpy(keys).cuda()
    d_ids = torch.empty(n, dtype=torch.int32, device="cuda")
    t.quantize_f32_device(n, d_keys.data_ptr(), d_ids.data_ptr(), v3dm_mod.LEAF_LOCAL)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_ids.cpu().numpy(), exp_local)
    replays = t.replays()
    print(f"BF {bf} depth {depth}: {replays} of {3 * n * depth} key-levels replayed in sequential order")
    assert replays < 3 * n * depth * 0.05  # near ties are rare; the fast pass decides the rest
    t.close()


def test_float_keys_on_a_byte_tree_and_near_ties(v3dm_mod, oracle_mod):
    """Float keys against a tree given as bytes (u/512), and children that differ by one ulp or
    not at all, so that the fast pass cannot decide and the sequential replay must."""
    bf, depth = 10, 3
    rng = synth.rng_for(77)
    nodes_u8 = synth.sift_like(rng, v3dm_mod.voctree_counts(bf, depth)[0])
    keys = synth.unit_sift(rng, 30000)
    exp = _ref_or_port(oracle_mod, bf, depth, nodes_u8.astype(np.float32) / 512, keys)
    t = v3dm_mod.VocabularyTreeTraversal(bf, depth)
    t.allocate(keys.shape[0])
    t.set_nodes(nodes_u8)
    np.testing.assert_array_equal(t.traverse_tree(keys, v3dm_mod.LEAF_LOCAL), exp)
    t.close()
    # near ties: children 1 and 2 of every node copy child 0, child 2 nudged by one ulp in one value
    nodes = synth.unit_sift(rng, v3dm_mod.voctree_counts(bf, depth)[0])
    nb = nodes.reshape(-1, bf, 128)
    nb[:, 1] = nb[:, 0]
    nb[:, 2] = nb[:, 0]
    nb[:, 2, 5] = np.nextafter(nb[:, 2, 5], np.float32(1))
    nodes = nb.reshape(-1, 128)
    exp = _ref_or_port(oracle_mod, bf, depth, nodes, keys)
    t = v3dm_mod.VocabularyTreeTraversal(bf, depth)
    t.allocate(keys.shape[0])
    t.set_nodes(nodes)
    np.testing.assert_array_equal(t.traverse_tree(keys, v3dm_mod.LEAF_LOCAL), exp)
    assert t.replays() > 0
    t.close()


def test_config_tree_all_queries(v3dm_mod, oracle_mod):
    """The vocabulary-tree configuration at full size: BF 10, depth 6, HKM centres from 500k
    descriptors, all 2,000,000 queries; leaf ids equal the reference CPU tree's."""
    nodes, keys = synth.voctree(3, 10, 6, 500_000, 2_000_000)
    t = v3dm_mod.VocabularyTreeTraversal(10, 6)
    t.allocate(keys.shape[0])
    t.set_nodes(nodes)
    got = t.traverse_tree(keys, v3dm_mod.LEAF_LOCAL)
    t.close()
    if oracle_mod.ref_voctree_available():
        exp = oracle_mod.ref_voctree(10, 6, nodes.astype(np.float32) / 512, keys.astype(np.float32) / 512)
    else:
        exp = oracle_mod.voctree(10, 6, nodes, keys, False)
    np.testing.assert_array_equal(got, exp)


def test_device_calls_reject_misaligned_buffers(v3dm_mod):
    """The device entry points read keys as 16-byte vectors and write int32 ids: misaligned
    buffers are an argument error, not a device fault."""
    import ctypes as C
    import torch
    dev = torch.device("cuda", 0)
    bf, depth, n = 4, 3, 100
    nodes = synth.sift_like(synth.rng_for(9), v3dm_mod.voctree_counts(bf, depth)[0])
    keys = torch.from_numpy(synth.sift_like(synth.rng_for(10), n + 1)).to(dev)
    ids = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    with v3dm_mod.VocabularyTreeTraversal(bf, depth) as t:
        t.allocate(n)
        t.set_nodes(nodes)
        L = v3dm_mod.lib()
        base_k, base_i = keys.data_ptr(), ids.data_ptr()
        assert L.v3dm_voctree_quantize_u8_device(t._h, n, C.c_void_p(base_k), C.c_void_p(base_i), 0) == v3dm_mod.OK
        for dk, di in ((base_k + 8, base_i), (base_k + 1, base_i), (base_k, base_i + 2)):
            st = L.v3dm_voctree_quantize_u8_device(t._h, n, C.c_void_p(dk), C.c_void_p(di), 0)
            assert st == v3dm_mod.ERR_ARG, (dk - base_k, di - base_i)
        fk = torch.zeros((n + 1) * 128 + 4, dtype=torch.float32, device=dev)
        st = L.v3dm_voctree_quantize_f32_device(t._h, n, C.c_void_p(fk.data_ptr() + 4), C.c_void_p(base_i), 0)
        assert st == v3dm_mod.ERR_ARG
        torch.cuda.synchronize()
