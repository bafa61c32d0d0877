"""GPU forward, loss and gradient kernels of the learned projection against the float64 CPU
restatement (oracle/projection.py), and training on matched pairs."""
import numpy as np
import pytest

from oracle import projection as P
from v3dm import synth

pytestmark = pytest.mark.gpu


def _pairs(seed, B, sigma=8.0):
    rng = synth.rng_for(seed)
    a = synth.sift_like(rng, B)
    return a, synth.noisy_copy(rng, a, sigma)


@pytest.mark.parametrize("B,T", [(16, 0.1), (256, 0.05), (1024, 0.07)])
def test_loss_and_gradient_equal_oracle(v3dm_mod, B, T):
    a, p = _pairs(B, B)
    net = v3dm_mod.Projection(seed=7)
    w = P.init_params(11)
    net.set_params(w)
    np.testing.assert_array_equal(net.params(), w)
    loss, g = net.loss_grad(a, p, T)
    ref_loss, ref_g = P.loss_grad(w, a, p, T)
    # FP32 accumulation against float64: relative 1e-4 on the loss, gradient entries within
    # 2e-3 of the largest gradient magnitude of their block
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-6
    for lo, hi in ((0, P.OFF_B1), (P.OFF_B1, P.OFF_W2), (P.OFF_W2, P.OFF_B2), (P.OFF_B2, P.N_PARAMS)):
        scale = np.abs(ref_g[lo:hi]).max()
        np.testing.assert_allclose(g[lo:hi], ref_g[lo:hi], rtol=0, atol=2e-3 * scale)
    net.close()


def test_embedding_and_cells_equal_oracle(v3dm_mod):
    rng = synth.rng_for(3)
    d = synth.sift_like(rng, 3000)
    net = v3dm_mod.Projection(seed=1)
    w = P.init_params(5)
    net.set_params(w)
    z = net.embed(d)
    zr = P.embed(w, d)
    np.testing.assert_allclose(z, zr, rtol=0, atol=2e-5)
    cents = zr[rng.choice(3000, 16, replace=False)].astype(np.float32)
    net.set_cells(cents)
    got = net.assign(d, 3)
    s = zr @ cents.astype(np.float64).T
    top = np.argsort(-s, axis=1, kind="stable")[:, :3]
    # identical except where two cell scores are within float rounding of each other
    srt = -np.sort(-s, axis=1)
    close = (srt[:, 0:3] - srt[:, 1:4]).min(1) < 1e-5
    assert np.mean(close) < 0.01
    np.testing.assert_array_equal(got[~close], top[~close])
    net.close()


def test_training_lowers_the_loss(v3dm_mod):
    import torch
    a, p = _pairs(9, 8192, sigma=12.0)
    da = torch.from_numpy(a).cuda()
    dp = torch.from_numpy(p).cuda()
    net = v3dm_mod.Projection(seed=2)
    B, T = 1024, 0.07
    first = net.loss_grad(a[:B], p[:B], T)[0]
    g = torch.Generator(device="cpu").manual_seed(0)
    for step in range(150):
        idx = torch.randperm(8192, generator=g)[:B].cuda()
        xa, xp = da[idx].contiguous(), dp[idx].contiguous()
        net.train_step(xa.data_ptr(), xp.data_ptr(), B, T, 3e-3)
    torch.cuda.synchronize()
    last = net.loss_grad(a[:B], p[:B], T)[0]
    assert last < 0.5 * first, (first, last)
    # the trained network ranks every anchor's own positive first among the batch's positives
    za, zp = net.embed(a[:B]), net.embed(p[:B])
    top1 = np.argmax(za @ zp.T, axis=1)
    assert np.mean(top1 == np.arange(B)) > 0.99
    net.close()
