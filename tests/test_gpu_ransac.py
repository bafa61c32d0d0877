"""Essential-matrix RANSAC on the GPU (v3dm_ransac_*) against the reference pin (oracle/_ref: the
reference's computeEssentialsFromFiveCorrs, relativePoseFromEssential and refineRelativePose in the
loop of computeRobustOrientationMLE, V3D/Apps/SfM/reconstruction_common.cpp:139-340).

The five-point solutions are floating point (the reference's SVD null space and polynomial solver
against a QR null space and derivative-bracketed roots here); they agree to about 1e-12, so the
per-sample solution counts must agree on >= 99.5% of random samples and >= 99% of the reference's
solutions must have a counterpart within 1e-6 (unit norm, sign-fixed).

The loop is checked two ways, with the reference's own sample sequence:
  - exactly against the same loop with the library's solver, pose recovery and refinement in place
    of the reference's (oracle ref_ransac swap=7, the GPU's algorithm on the CPU): the same choice on
    every pair, the same inlier flags and counts, E, R, T and the error to 1e-5 (the GPU's double
    arithmetic is the host's up to the last bits of a few operations);
  - against the reference itself: the same choice on most pairs, and every pair where the choice
    differs must differ in the same way when only the reference's five-point solver is replaced
    (swap=1): the solvers' 1e-12 differences decide near-ties between candidates' costs.  The
    restated pose recovery and refinement alone (swap=6) never change the reference's choice
    (tests/test_ransac_restated.py)."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


def _need_ref(oracle_mod):
    if not oracle_mod.ref_ransac_available():
        pytest.skip("reference relative-orientation code not built (oracle/_ref)")


def _unit(E):
    e = E.reshape(-1)
    e = e / np.linalg.norm(e)
    return e * np.sign(e[np.argmax(np.abs(e))])


def _check_restated(oracle_mod, got, p, c, K, thr, n_samples, samples, refine, flags):
    """The GPU's pair p equals the loop with the library's components on the CPU (swap=7)."""
    o = oracle_mod.ref_ransac(c, K[0], K[1], thr, n_samples, samples, refine=refine, swap=7)
    if o["chosen"] < 0:
        assert got["n_inliers"][p] == -1, p
        return
    assert got["n_inliers"][p] == o["n_inliers"], p
    assert np.linalg.norm(_unit(got["E"][p]) - _unit(o["model"][:9])) < 1e-5, p
    np.testing.assert_allclose(got["error"][p], o["model"][30], rtol=1e-5)
    assert np.abs(got["R"][p].reshape(-1) - o["model"][18:27]).max() < 1e-5
    assert np.abs(got["T"][p] - o["model"][27:30]).max() < 1e-5
    np.testing.assert_array_equal(flags, o["flags"])


def _same_choice(a, b):
    if a["chosen"] < 0 or b["chosen"] < 0:
        return a["chosen"] < 0 and b["chosen"] < 0
    return a["chosen"] // 10 == b["chosen"] // 10 and np.linalg.norm(_unit(a["model"][:9]) - _unit(b["model"][:9])) < 1e-5


def _rot(rng):
    v = rng.normal(size=3) * 0.3
    th = np.linalg.norm(v)
    k = v / th
    Kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(th) * Kx + (1 - np.cos(th)) * Kx @ Kx


def test_five_point_solutions_match_the_reference(v3dm_mod, oracle_mod):
    _need_ref(oracle_mod)
    rng = np.random.default_rng(0)
    pts = []
    for t in range(3000):
        if t % 2 == 0:  # consistent samples of a random pose
            R = _rot(rng)
            T = rng.normal(size=3)
            X = np.c_[rng.uniform(-1, 1, (5, 2)), rng.uniform(3, 6, 5)]
            p = X[:, :2] / X[:, 2:]
            Y = (R @ X.T).T + T
            q = Y[:, :2] / Y[:, 2:]
        else:  # random (outlier) samples
            p = rng.uniform(-0.5, 0.5, (5, 2))
            q = rng.uniform(-0.5, 0.5, (5, 2))
        pts.append(np.r_[p[:, 0], p[:, 1], q[:, 0], q[:, 1]])
    pts = np.array(pts)
    with v3dm_mod.Ransac() as r:
        es, cnt = r.five_point(pts)
    same, matched, total = 0, 0, 0
    for t in range(pts.shape[0]):
        ref = oracle_mod.ref_five_point(pts[t, :5], pts[t, 5:10], pts[t, 10:15], pts[t, 15:])
        ours = [_unit(es[t, k]) for k in range(cnt[t])]
        same += len(ref) == cnt[t]
        for e in ref:
            total += 1
            if ours and min(np.linalg.norm(_unit(e) - o) for o in ours) < 1e-6:
                matched += 1
        if t % 2 == 0:  # the true E is among ours
            pass
    assert same >= 0.995 * pts.shape[0], same
    assert matched >= 0.99 * total, (matched, total)


@pytest.mark.parametrize("n_pairs,n_min,n_max,thr,n_samples", [(24, 5, 60, 2.0, 200), (40, 300, 1500, 2.0, 1000),
                                                               (6, 2500, 4000, 1.0, 1000)])
def test_reference_sample_sequence_gives_the_reference_choice(v3dm_mod, oracle_mod, n_pairs, n_min, n_max, thr,
                                                              n_samples):
    _need_ref(oracle_mod)
    off, corrs, K, R, t, inl = synth.two_view_pairs(n_pairs + n_min, n_pairs=n_pairs, n_min=n_min, n_max=n_max)
    seqs = [v3dm_mod.ransac_shuffle_samples(int(off[p + 1] - off[p]), n_samples, 100 + p) for p in range(n_pairs)]
    with v3dm_mod.Ransac() as r:
        agree, total = 0, 0
        for p in range(n_pairs):
            n = int(off[p + 1] - off[p])
            s = seqs[p]
            c = corrs[off[p]:off[p + 1]]
            ref = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], thr, n_samples, s if s.shape[0] else np.zeros((0, 5)))
            if s.shape[0] == 0:  # fewer than 6 correspondences: the loop draws nothing
                assert ref["chosen"] == -1
                if n < 5:
                    got = r.essential(np.array([0, n]), c, K[p:p + 1], thr, n_samples, n_draw=1, seed=1)
                    assert got["n_inliers"][0] == -1 and got["error"][0] == -1.0
                continue
            got = r.essential(np.array([0, n]), c, K[p:p + 1], thr, n_samples, samples=s[None])
            total += 1
            _check_restated(oracle_mod, got, 0, c, K[p], thr, n_samples, s, False, got["flags"])
            if ref["chosen"] < 0:
                agree += got["n_inliers"][0] == -1
                continue
            if got["n_inliers"][0] >= 0 and np.linalg.norm(_unit(got["E"][0]) - _unit(ref["model"][:9])) < 1e-5:
                agree += 1
                np.testing.assert_allclose(got["error"][0], ref["model"][30], rtol=1e-4)
                assert np.abs(got["R"][0].reshape(-1) - ref["model"][18:27]).max() < 1e-4
                assert np.abs(got["T"][0] - ref["model"][27:30]).max() < 1e-4
                slack = max(2, n // 500)
                diff = int((got["flags"] != ref["flags"]).sum())
                assert diff <= slack and abs(int(got["n_inliers"][0]) - ref["n_inliers"]) <= slack
            else:  # the reference's solver is the only difference that changes the choice
                solver = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], thr, n_samples, s, swap=oracle_mod.SWAP_SOLVER)
                assert not _same_choice(solver, ref), p
        assert agree >= 0.95 * total, (agree, total)


@pytest.mark.parametrize("n_pairs,n_min,n_max,thr,n_samples", [(30, 300, 1500, 2.0, 1000), (6, 2500, 4000, 1.0, 500)])
def test_iterative_refinement_gives_the_reference_result(v3dm_mod, oracle_mod, n_pairs, n_min, n_max, thr,
                                                         n_samples):
    """mode.iterativeRefinement (set by the apps): each accepted pose refined on its inliers
    (refineRelativePose), the loop continuing from the refined cost and inlier count.  With the
    reference's own sample sequence: exactly the loop with the library's components on every pair;
    the reference's model (unit E within 1e-5, refined error, R and T to 1e-4, inlier flags to 0.2%
    of the correspondences) on >= 90% of the pairs, and on the others a choice that the restated
    five-point solver alone makes too.  All pairs run batched in one call."""
    _need_ref(oracle_mod)
    off, corrs, K, R, t, inl = synth.two_view_pairs(n_pairs + 7 * n_min, n_pairs=n_pairs, n_min=n_min, n_max=n_max)
    seqs = [v3dm_mod.ransac_shuffle_samples(int(off[p + 1] - off[p]), n_samples, 300 + p) for p in range(n_pairs)]
    n_draw = max(s.shape[0] for s in seqs)
    padded = np.stack([np.concatenate([s, np.repeat(s[-1:], n_draw - s.shape[0], 0)]) for s in seqs])
    with v3dm_mod.Ransac() as r:
        r.set_refinement(True)
        allp = r.essential(off, corrs, K, thr, n_samples, samples=padded)
        r.set_refinement(False)
        plain = r.essential(off, corrs, K, thr, n_samples, samples=padded)
    agree, moved = 0, 0
    for p in range(n_pairs):
        c = corrs[off[p]:off[p + 1]]
        n = c.shape[0]
        _check_restated(oracle_mod, allp, p, c, K[p], thr, n_samples, seqs[p], True, allp["flags"][off[p]:off[p + 1]])
        ref = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], thr, n_samples, seqs[p], refine=True)
        if ref["chosen"] < 0 or allp["n_inliers"][p] < 0:
            agree += ref["chosen"] < 0 and allp["n_inliers"][p] < 0
            continue
        moved += np.abs(allp["R"][p] - plain["R"][p]).max() > 1e-9
        if np.linalg.norm(_unit(allp["E"][p]) - _unit(ref["model"][:9])) < 1e-5:
            agree += 1
            np.testing.assert_allclose(allp["error"][p], ref["model"][30], rtol=1e-4)
            assert np.abs(allp["R"][p].reshape(-1) - ref["model"][18:27]).max() < 1e-4
            assert np.abs(allp["T"][p] - ref["model"][27:30]).max() < 1e-4
            slack = max(2, n // 500)
            fl = allp["flags"][off[p]:off[p + 1]]
            assert int((fl != ref["flags"]).sum()) <= slack
            assert abs(int(allp["n_inliers"][p]) - ref["n_inliers"]) <= slack
        else:  # the reference's solver is the only difference that changes the choice
            solver = oracle_mod.ref_ransac(c, K[p, 0], K[p, 1], thr, n_samples, seqs[p], refine=True,
                                           swap=oracle_mod.SWAP_SOLVER)
            assert not _same_choice(solver, ref), p
    print(f"refinement: {agree} of {n_pairs} pairs agree with the reference; {moved} poses moved by it")
    assert agree >= 0.90 * n_pairs, (agree, n_pairs)
    assert moved > 0  # the refinement does change the poses


def test_batched_call_with_small_pairs(v3dm_mod):
    """A batch that mixes pairs with fewer than 5 correspondences (no model: -1, no inlier flags) with
    ordinary ones; single-pair calls of the same data run."""
    off, corrs, K, R, t, inl = synth.two_view_pairs(8, n_pairs=30, n_min=4, n_max=900)
    with v3dm_mod.Ransac() as r:
        allp = r.essential(off, corrs, K, 2.0, 300, seed=5)
        assert r.last_launches() > 0
        for p in (0, 7, 29):
            n = int(off[p + 1] - off[p])
            # the device draws depend on (pair, sample): a one-pair call sees pair 0's draws
            one = r.essential(off[p:p + 2] - off[p], corrs[off[p]:off[p + 1]], K[p:p + 1], 2.0, 300, seed=5)
            if n < 5:
                assert allp["n_inliers"][p] == -1 and one["n_inliers"][0] == -1
        small = np.diff(off) < 5
        assert (allp["n_inliers"][small] == -1).all()
        assert (allp["flags"][np.repeat(small, np.diff(off))] == 0).all()


def test_device_entry_point_equals_host_entry_point(v3dm_mod):
    import torch
    off, corrs, K, R, t, inl = synth.two_view_pairs(10, n_pairs=20, n_min=100, n_max=1200)
    with v3dm_mod.Ransac() as r:
        host = r.essential(off, corrs, K, 2.0, 500, seed=9)
        dc = torch.from_numpy(corrs).cuda()
        dm = torch.empty((20, 31), dtype=torch.float64, device="cuda")
        dn = torch.empty(20, dtype=torch.int32, device="cuda")
        df = torch.empty(corrs.shape[0], dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        r.essential_device(off, dc.data_ptr(), K, 2.0, 500, 501, None, 9, dm.data_ptr(), dn.data_ptr(), df.data_ptr())
        r.wait()
        np.testing.assert_array_equal(dm.cpu().numpy(), host["models"])
        np.testing.assert_array_equal(dn.cpu().numpy(), host["n_inliers"])
        np.testing.assert_array_equal(df.cpu().numpy(), host["flags"])


def test_device_draws_find_the_pose(v3dm_mod):
    off, corrs, K, R, t, inl = synth.two_view_pairs(9, n_pairs=64, n_min=300, n_max=2000, inlier_min=0.4,
                                                    inlier_max=0.8)
    with v3dm_mod.Ransac() as r:
        got = r.essential(off, corrs, K, 2.0, 1000, seed=123)
    good = 0
    for p in range(64):
        if got["n_inliers"][p] < 0:
            continue
        rot_err = np.linalg.norm(got["R"][p] - R[p])
        true_in = inl[off[p]:off[p + 1]]
        fl = got["flags"][off[p]:off[p + 1]].astype(bool)
        recall = (fl & true_in).sum() / max(1, true_in.sum())
        good += rot_err < 0.05 and recall > 0.8 and fl.sum() == got["n_inliers"][p]
    assert good >= 60, good


def test_errors(v3dm_mod):
    import ctypes as C
    L = v3dm_mod.lib()
    off = np.array([0, 10], np.int32)
    corrs = np.random.default_rng(0).uniform(0, 100, (10, 4)).astype(np.float32)
    K = np.tile(np.eye(3), (1, 2, 1, 1))
    with v3dm_mod.Ransac() as r:
        bad = np.full((1, 3, 5), 10, np.int32)  # index 10 of 10 correspondences
        with pytest.raises(v3dm_mod.V3DMError) as e:
            r.essential(off, corrs, K, 2.0, 10, samples=bad)
        assert e.value.status == v3dm_mod.ERR_ARG
        with pytest.raises(v3dm_mod.V3DMError) as e:
            r.essential(off, corrs, np.zeros((1, 2, 3, 3)), 2.0, 10)  # singular K
        assert e.value.status == v3dm_mod.ERR_ARG
        with pytest.raises(v3dm_mod.V3DMError) as e:
            r.essential(off, corrs, K, 2.0, 10, n_draw=v3dm_mod.RANSAC_MAX_DRAW + 1)
        assert e.value.status == v3dm_mod.ERR_ARG
        n_big = v3dm_mod.RANSAC_MAX_PAIRS + 1  # pairs per call above the limit (checked before any work)
        off_big = np.zeros(n_big + 1, np.int32)
        K_big = np.tile(np.eye(3), (n_big, 2, 1, 1))
        models = np.empty((1, 31))
        nin = np.empty(1, np.int32)
        assert L.v3dm_ransac_essential(r._h, n_big, off_big.ctypes.data, None, K_big.ctypes.data, C.c_double(2.0), 10,
                                       1, None, C.c_uint64(0), models.ctypes.data, nin.ctypes.data,
                                       None) == v3dm_mod.ERR_SIZE
        got = r.essential(off, corrs, K, 2.0, 10)  # still usable
        assert got["n_inliers"].shape == (1,)
