"""Essential-matrix RANSAC, CPU part: the library's sample sequence (v3dm_ransac_shuffle_samples,
host code) against the reference loop's own draws (srand, std::random_shuffle, consecutive
5-tuples: V3D/Apps/SfM/reconstruction_common.cpp:110-114, 173-205), and the reference pin itself
(oracle/_ref: the reference's five-point solver and pose recovery in the loop of
computeRobustOrientationMLE) on synthetic two-view data."""
import numpy as np
import pytest

from v3dm import synth


@pytest.mark.parametrize("n,n_samples,seed", [(4, 1000, 1), (5, 1000, 1), (6, 1000, 2), (9, 10, 3), (137, 1000, 4),
                                              (800, 1000, 5), (5000, 1000, 6), (300, 0, 7)])
def test_samples_equal_the_reference_draws(v3dm_mod, oracle_mod, n, n_samples, seed):
    if not oracle_mod.ref_ransac_available():
        pytest.skip("reference relative-orientation code not built (oracle/_ref)")
    got = v3dm_mod.ransac_shuffle_samples(n, n_samples, seed)
    exp = oracle_mod.ref_shuffle_samples(n, n_samples, seed)
    np.testing.assert_array_equal(got, exp)
    if n >= 6:
        assert got.shape[0] == min(n_samples + 1, max(1, int(n_samples * 5.0 / n + 0.5)) * ((n - 5 + 4) // 5))
        assert (got >= 0).all() and (got < n).all()
        assert all(len(set(r)) == 5 for r in got)


def test_reference_pin_recovers_the_pose(oracle_mod):
    if not oracle_mod.ref_ransac_available():
        pytest.skip("reference relative-orientation code not built (oracle/_ref)")
    off, corrs, K, R, t, inl = synth.two_view_pairs(3, n_pairs=3, n_min=400, n_max=600, inlier_min=0.6,
                                                    inlier_max=0.7)
    for p in range(3):
        c = corrs[off[p]:off[p + 1]]
        smp = oracle_mod.ref_shuffle_samples(c.shape[0], 1000, 11 + p)
        res = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], 2.0, 1000, smp)
        assert res["chosen"] >= 0
        Rm = res["model"][18:27].reshape(3, 3)
        assert np.linalg.norm(Rm - R[p]) < 0.05
        flags = res["flags"].astype(bool)
        assert flags.sum() == res["n_inliers"]
        assert (flags & inl[off[p]:off[p + 1]]).sum() > 0.8 * inl[off[p]:off[p + 1]].sum()


def test_sampler_capacity_and_errors(v3dm_mod):
    import ctypes as C
    L = v3dm_mod.lib()
    full = v3dm_mod.ransac_shuffle_samples(50, 100, 9)
    out = np.full((10, 5), -7, np.int32)
    nd = C.c_int(-1)
    # a short buffer: the first 'cap' samples, V3DM_ERR_CAPACITY
    assert L.v3dm_ransac_shuffle_samples(50, 100, 9, 10, out.ctypes.data, C.byref(nd)) == v3dm_mod.ERR_CAPACITY
    assert nd.value == 10
    np.testing.assert_array_equal(out, full[:10])
    assert L.v3dm_ransac_shuffle_samples(4, 100, 9, 10, out.ctypes.data, C.byref(nd)) == v3dm_mod.OK
    assert nd.value == 0
    assert L.v3dm_ransac_shuffle_samples(-1, 100, 9, 10, out.ctypes.data, C.byref(nd)) == v3dm_mod.ERR_ARG
    assert L.v3dm_ransac_shuffle_samples(50, 100, 9, 10, None, C.byref(nd)) == v3dm_mod.ERR_ARG


def _fixture():
    from pathlib import Path
    return np.load(Path(__file__).resolve().parent / "golden" / "ransac_ref.npz")


def test_sampler_equals_the_fixture_draws(v3dm_mod):
    """The committed fixture holds the reference's own draws (srand + std::random_shuffle); the
    library's sampler reproduces them without the reference build."""
    z = _fixture()
    off = z["rs_offsets"]
    for p in range(6):
        got = v3dm_mod.ransac_shuffle_samples(int(off[p + 1] - off[p]), 1000, int(z["rs_seeds"][p]))
        np.testing.assert_array_equal(got, z[f"rs_samples_{p}"])


def test_reference_pin_reproduces_the_fixture(oracle_mod):
    if not oracle_mod.ref_ransac_available():
        pytest.skip("reference relative-orientation code not built (oracle/_ref)")
    z = _fixture()
    pts, E, cnt = z["fp_pts"], z["fp_E"], z["fp_counts"]
    for t in range(0, pts.shape[0], 7):
        got = oracle_mod.ref_five_point(pts[t, :5], pts[t, 5:10], pts[t, 10:15], pts[t, 15:])
        assert len(got) == cnt[t]
        np.testing.assert_array_equal(got, E[t, :cnt[t]])
    off, corrs, K = z["rs_offsets"], z["rs_corrs"], z["rs_K"]
    for p in range(6):
        res = oracle_mod.ref_ransac(corrs[off[p]:off[p + 1]], K[p, 0], K[p, 1], 2.0, 1000, z[f"rs_samples_{p}"])
        assert res["chosen"] == z["rs_chosen"][p] and res["n_inliers"] == z["rs_n_inliers"][p]
        np.testing.assert_array_equal(res["model"], z["rs_models"][p])
        np.testing.assert_array_equal(res["flags"], z["rs_flags"][off[p]:off[p + 1]])


def test_reference_pin_with_refinement(oracle_mod):
    """The pin's refined mode (the apps' mode.iterativeRefinement: the reference's
    refineRelativePose on each accepted pose) runs and keeps the pose; the default mode is the
    fixture's."""
    if not oracle_mod.ref_ransac_available():
        pytest.skip("reference relative-orientation code not built (oracle/_ref)")
    off, corrs, K, R, t, inl = synth.two_view_pairs(12, n_pairs=3, n_min=300, n_max=700, inlier_min=0.5,
                                                    inlier_max=0.7)
    for p in range(3):
        c = corrs[off[p]:off[p + 1]]
        smp = oracle_mod.ref_shuffle_samples(c.shape[0], 1000, 40 + p)
        plain = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], 2.0, 1000, smp)
        refined = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], 2.0, 1000, smp, refine=True)
        assert refined["chosen"] >= 0 and plain["chosen"] >= 0
        assert np.linalg.norm(refined["model"][18:27].reshape(3, 3) - R[p]) < 0.05
        assert refined["model"][30] <= plain["model"][30] * 1.05


def test_padding_with_the_last_sample_keeps_the_choice(oracle_mod):
    """The reference loop on a short sample sequence and on the same sequence padded with repeats of
    its last sample gives the same result (the padding the C++ wrapper and batched calls use)."""
    if not oracle_mod.ref_ransac_available():
        pytest.skip("reference relative-orientation code not built (oracle/_ref)")
    off, corrs, K, R, t, inl = synth.two_view_pairs(13, n_pairs=4, n_min=8, n_max=40, inlier_min=0.4,
                                                    inlier_max=0.9)
    for p in range(4):
        c = corrs[off[p]:off[p + 1]]
        s = oracle_mod.ref_shuffle_samples(c.shape[0], 1000, 60 + p)
        assert 0 < s.shape[0] < 1001  # short: few correspondences
        padded = np.concatenate([s, np.repeat(s[-1:], 1001 - s.shape[0], axis=0)])
        a = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], 2.0, 1000, s)
        b = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], 2.0, 1000, padded)
        assert a["chosen"] == b["chosen"] and a["n_inliers"] == b["n_inliers"]
        np.testing.assert_array_equal(a["model"], b["model"])
