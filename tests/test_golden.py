"""Golden fixtures made by the reference's own code (tests/golden/make_golden.py).

voctree_ref.npz: leaf-local ids from the reference's CPU vocabulary tree
(V3D/Base/v3d_vocabularytree.h getVisualWord).  match_ref.npz: (left, right) pairs from the
reference's CUDA SIFT_Matching (V3D/CUDA/v3d_cudamatching.cu) run on a B200.  The CPU tests pin
the oracle to them; the GPU tests hold the CUDA path to them through the C ABI."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _load(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.fail(f"{p} missing: regenerate with tests/golden/make_golden.py")
    return np.load(p)


def _voctree_cases():
    d = _load("voctree_ref.npz")
    for i in range(int(d["n_cases"])):
        bf, depth = (int(x) for x in d[f"c{i}_shape"])
        yield bf, depth, d[f"c{i}_nodes"], d[f"c{i}_keys"], d[f"c{i}_leaf_local"]


def _match_cases():
    d = _load("match_ref.npz")
    for i in range(int(d["n_cases"])):
        inp = str(d[f"c{i}_input"])
        ms, mr = (float(x) for x in d[f"c{i}_params"])
        gates = []
        for g in d[f"c{i}_gates"]:
            t, thr = str(g).split(":")
            gates.append((t, d[f"{inp}_{t}"], float(thr)))
        kw = {}
        if gates:
            kw = dict(lpos=d[f"{inp}_lpos"], rpos=d[f"{inp}_rpos"])
        yield i, d[f"{inp}_L"], d[f"{inp}_R"], ms, mr, gates, kw, d[f"c{i}_pairs"]


def _level_start(bf, depth):
    return sum(bf ** d for d in range(1, depth))


def test_oracle_voctree_equals_reference_fixture(oracle_mod):
    n = 0
    for bf, depth, nodes, keys, ids in _voctree_cases():
        np.testing.assert_array_equal(oracle_mod.voctree(bf, depth, nodes, keys, False), ids)
        np.testing.assert_array_equal(oracle_mod.voctree(bf, depth, nodes, keys, True), ids + _level_start(bf, depth))
        np.testing.assert_array_equal(
            oracle_mod.voctree(bf, depth, nodes.astype(np.float32) / 512, keys.astype(np.float32) / 512, False), ids)
        n += 1
    assert n >= 6


def test_oracle_match_equals_reference_fixture(oracle_mod):
    n = 0
    for i, L, R, ms, mr, gates, kw, pairs in _match_cases():
        got = oracle_mod.match(L, R, ms, mr, gates=gates, **kw)
        np.testing.assert_array_equal(got, pairs, err_msg=f"case {i}")
        n += 1
    assert n >= 10


def test_match_fixture_covers_the_edge_cases():
    d = _load("match_ref.npz")
    kinds = {(str(d[f"c{i}_input"]), float(d[f"c{i}_params"][1]) < 0, len(d[f"c{i}_gates"]))
             for i in range(int(d["n_cases"]))}
    assert ("pair", True, 0) in kinds  # no-ratio path
    assert ("stereo", False, 2) in kinds  # compounding gates
    assert ("ties", False, 0) in kinds
    L = d["ties_L"]
    assert np.array_equal(L[:64], L[128:192])  # duplicated lefts: ties in every right's best and second


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["tcgen05", "simt"])
def test_cuda_match_equals_reference_fixture(v3dm_mod, kernel):
    kern = v3dm_mod.KERNEL_TCGEN05 if kernel == "tcgen05" else v3dm_mod.KERNEL_SIMT
    m = v3dm_mod.SIFTMatching(0, kern)
    m.allocate(1024, 1024, True)
    for i, L, R, ms, mr, gates, kw, pairs in _match_cases():
        m.set_left_features(L)
        m.set_right_features(R)
        got = m.find_putative_matches(ms, mr)
        for t, M, thr in gates:
            if t == "F":
                got = m.run_guided_matching(M, thr, kw["lpos"], kw["rpos"], ms, mr)
            else:
                got = m.run_guided_homography_matching(M, thr, kw["lpos"], kw["rpos"], ms, mr)
        np.testing.assert_array_equal(got, pairs, err_msg=f"case {i} ({kernel})")
    m.close()


@pytest.mark.gpu
def test_cuda_voctree_equals_reference_fixture(v3dm_mod):
    for bf, depth, nodes, keys, ids in _voctree_cases():
        t = v3dm_mod.VocabularyTreeTraversal(bf, depth)
        t.allocate(keys.shape[0])
        t.set_nodes(nodes)
        np.testing.assert_array_equal(t.traverse_tree(keys, v3dm_mod.LEAF_LOCAL), ids)
        np.testing.assert_array_equal(t.traverse_tree(keys, v3dm_mod.LEAF_GLOBAL), ids + _level_start(bf, depth))
        t.close()
