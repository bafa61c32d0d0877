"""Candidate-proposal matching (v3dm_batch_match_proposal) on the GPU.

Pass A of the proposal applies the reference's column rule (v3d_cudamatching.cu:133-162) to the
score matrix in which every non-candidate entry is masked (-1e20, as the guided gates mask): a
candidate is a (left, right) whose cells share a probed cell.  Each left it accepts is then
decided again on the full score matrix of its pair, and so is the right that exact decision
names (.cu:164-210); the pair is kept when the two name each other (.cu:546-551).  So the result
is the set of exhaustive matches whose left the masked pass accepted: a subset of exhaustive
matching.  That restatement (numpy, float32 per operation) is the checker; with every cell
probed the proposal must reproduce exhaustive matching exactly."""
import numpy as np
import pytest

from oracle import projection as P
from v3dm import proposal, synth

pytestmark = pytest.mark.gpu

f32 = np.float32


def _side(M, ms, mr):
    """Reference decisions of the rows of M (rows = the side deciding, columns = the other
    side; the same float32 operations as tests/pyref.py)."""
    n, m = M.shape
    if m == 0:
        return np.full(n, -1)
    arg = np.argmax(M, axis=1)  # first index on ties, as the strict '>' scan
    mx = M[np.arange(n), arg]
    if m > 1:
        srt = -np.sort(-M, axis=1)
        nxt = srt[:, 1]
    else:
        nxt = np.full(n, f32(-1e30), np.float32)
    if mr < 0:
        return np.where(mx > f32(ms), arg, -1)
    nextDist = np.maximum(0.001, (f32(2.0) - f32(2.0) * nxt).astype(np.float64)).astype(np.float32)
    bestDist = (f32(2.0) - f32(2.0) * mx).astype(np.float32)
    ratio = (bestDist / nextDist).astype(np.float32)
    return np.where((mx > f32(ms)) & (ratio < f32(mr)), arg, -1)


def _proposal_reference(L, R, mask, ms, mr):
    """Exhaustive matches (l, r) whose left the masked column rule accepts."""
    S = (R.astype(np.int64) @ L.astype(np.int64).T).astype(np.float32) * f32(2.0 ** -18)  # [r, l]
    masked = np.where(mask.T, S, f32(-1e20)).astype(np.float32)
    accepted = _side(masked.T, ms, mr) >= 0
    col = _side(S.T, ms, mr)  # exact, per left
    row = _side(S, ms, mr)    # exact, per right
    out = [(k, col[k]) for k in range(L.shape[0]) if accepted[k] and col[k] >= 0 and row[col[k]] == k]
    return np.array(out, np.int32).reshape(-1, 2)


def _exhaustive_reference(L, R, ms, mr):
    return _proposal_reference(L, R, np.ones((L.shape[0], R.shape[0]), bool), ms, mr)


def _images(seed, counts, track_frac=0.2):
    rng = synth.rng_for(seed)
    counts = np.asarray(counts, np.int64)
    base = synth.sift_like(rng, max(1, int(track_frac * counts.sum() / 3)))
    parts = []
    for c in counts:
        k = min(int(round(track_frac * c)), int(c))
        tr = rng.integers(0, base.shape[0], k)
        parts.append(np.concatenate([synth.noisy_copy(rng, base[tr]), synth.sift_like(rng, int(c) - k)]))
    desc = np.concatenate(parts)
    return desc, counts.astype(np.int32), np.concatenate([[0], np.cumsum(counts)])


@pytest.fixture(scope="module")
def small():
    return _images(21, [300, 257, 1, 0, 450, 129, 600, 64])


def _net_with_cells(v3dm_mod, desc, n_cells, seed=3):
    net = v3dm_mod.Projection(seed=seed)
    z = net.embed(desc)
    net.set_cells(proposal.fit_cells(z, n_cells, iters=10, seed=seed))
    return net


@pytest.mark.parametrize("probes,probes_right,ms,mr,n_cells,schedule",
                         [(1, 1, 0.7, 0.8, 6, 0), (2, 1, 0.7, 0.8, 6, 0), (3, 1, 0.6, 0.9, 6, 0),
                          (2, 1, 0.7, -1.0, 6, 0), (2, 2, 0.7, 0.8, 6, 0), (3, 2, 0.6, 0.9, 6, 0),
                          (1, 3, 0.7, 0.8, 6, 0), (2, 2, 0.7, 0.8, 6, 2), (3, 2, 0.6, 0.9, 6, 1),
                          (5, 6, 0.7, 0.8, 40, 2), (8, 8, 0.7, 0.8, 256, 2)])
def test_proposal_equals_masked_reference(v3dm_mod, small, probes, probes_right, ms, mr, n_cells, schedule):
    """Candidates: a left probing one of the cells a right probes (symmetric probing scores a
    pair once per shared cell; the result must not depend on it), for every row schedule."""
    desc, counts, offs = small
    net = _net_with_cells(v3dm_mod, desc, n_cells)
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    b.set_config(b.config()[0], schedule)
    per = b.split_pairs(b.match_proposal(net, probes, ms, mr, probes_right=probes_right))
    cells = net.assign(desc, max(probes, probes_right))
    pairs = synth.all_pairs(len(counts))
    for k, (i, j) in enumerate(pairs):
        ci, cj = cells[offs[i]:offs[i + 1], :probes], cells[offs[j]:offs[j + 1], :probes_right]
        mask = (ci[:, :, None, None] == cj[None, None, :, :]).any(axis=(1, 3))  # [left, right]
        Li, Rj = desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]]
        exp = _proposal_reference(Li, Rj, mask, ms, mr)
        np.testing.assert_array_equal(per[k], exp, err_msg=f"pair {k} ({i}, {j})")
        # precision 1: every pair it returns is a pair of exhaustive matching
        full = {tuple(x) for x in _exhaustive_reference(Li, Rj, ms, mr)}
        assert all(tuple(x) in full for x in per[k])
    scored, exhaustive = b.proposal_scored()
    assert 0 < scored <= exhaustive * min(probes, probes_right)  # once per shared cell
    b.close()
    net.close()


def test_all_cells_probed_equals_exhaustive(v3dm_mod):
    desc, counts, _ = _images(22, [1200, 2500, 700, 3000, 1800, 900])
    net = _net_with_cells(v3dm_mod, desc, 4)
    b = v3dm_mod.BatchMatching()
    b.set_images(desc, counts)
    b.set_pairs(None)
    exh = b.match(0.7, 0.8)
    got = b.match_proposal(net, 4, 0.7, 0.8)
    np.testing.assert_array_equal(got, exh)
    scored, exhaustive = b.proposal_scored()
    assert scored == exhaustive
    # every right listed under all 4 cells, every left probing 2: each pair is scored twice, in
    # two cell blocks, and the result is still exhaustive matching
    np.testing.assert_array_equal(b.match_proposal(net, 2, 0.7, 0.8, probes_right=4), exh)
    assert b.proposal_scored()[0] == 2 * exhaustive
    # graph replay and the graph-free path agree
    again = b.match_proposal(net, 4, 0.7, 0.8)
    b.use_graph(False)
    np.testing.assert_array_equal(again, exh)
    np.testing.assert_array_equal(b.match_proposal(net, 4, 0.7, 0.8), exh)
    b.close()
    net.close()


def test_trained_projection_gains_recall(v3dm_mod):
    """Held-out images give training pairs; on test images the cells of the trained network find
    more of the exhaustive matches than the same number of cells fitted to the untrained network
    (same seed), at the same number of probes."""
    tr_desc, tr_counts, tr_offs = synth.images(41, n_images=60, n_min=4000, n_max=4000)
    te_desc, te_counts, _ = synth.images(42, n_images=40, n_min=4000, n_max=4000)
    b = v3dm_mod.BatchMatching()
    b.set_images(tr_desc, tr_counts)
    b.set_pairs(None)
    a, p = proposal.mine_pairs(tr_desc, tr_offs, synth.all_pairs(len(tr_counts)), b.match(0.7, 0.8))
    assert a.shape[0] > 20000
    b.set_images(te_desc, te_counts)
    b.set_pairs(None)
    exh = b.match(0.7, 0.8)
    results = {}
    for trained in (False, True):
        net = v3dm_mod.Projection(seed=5)
        if trained:
            losses = proposal.train(net, a, p, steps=400, batch=2048, temperature=0.2, lr=2e-3)
            assert losses[-1][1] < losses[0][1]
        net.set_cells(proposal.fit_cells(net.embed(tr_desc), 16, seed=1))
        got = b.match_proposal(net, 4, 0.7, 0.8)
        results[trained] = proposal.recall(exh, got)
        net.close()
    assert results[True][0] > results[False][0], results
    assert results[True][0] > 0.85, results
    assert results[True][1] == 1.0 and results[False][1] == 1.0, results  # a subset of exhaustive matching
    b.close()


def test_gradients_of_trained_state_still_match_oracle(v3dm_mod):
    """After Adam steps the device parameters still give the oracle's loss and gradient."""
    import torch
    rng = synth.rng_for(8)
    a = synth.sift_like(rng, 512)
    p = synth.noisy_copy(rng, a, 8.0)
    net = v3dm_mod.Projection(seed=9)
    da, dp = torch.from_numpy(a).cuda(), torch.from_numpy(p).cuda()
    for _ in range(5):
        net.train_step(da.data_ptr(), dp.data_ptr(), 512, 0.05, 1e-3)
    torch.cuda.synchronize()
    w = net.params()
    loss, g = net.loss_grad(a[:256], p[:256], 0.05)
    ref_loss, ref_g = P.loss_grad(w, a[:256], p[:256], 0.05)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss)
    np.testing.assert_allclose(g, ref_g, rtol=0, atol=2e-3 * np.abs(ref_g).max())
    net.close()
