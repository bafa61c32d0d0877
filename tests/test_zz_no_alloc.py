"""v3dm_putative_u8_noalloc: putative matching that allocates no device memory.

It serves callers that cannot allocate device memory mid-run (a host application that owns
all GPU memory, a frame loop where an allocation would synchronise the device).  This file
is collected last so that a run stopping at the first failure has already run every other
test.  It calls the entry point through the C ABI twice in a row, on different inputs, and
requires the same pairs as the allocating entry point v3dm_putative (bit-exact: pair
indices are integers)."""
import ctypes as C

import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


def _entry(v3dm_mod):
    fn = v3dm_mod.lib().v3dm_putative_u8_noalloc
    fn.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def test_noalloc_matches_allocating_entry_point_twice(v3dm_mod):
    import torch
    dev = torch.device("cuda", 0)
    fn = _entry(v3dm_mod)
    stream = torch.cuda.current_stream(dev)
    for seed, nL, nR in ((11, 3000, 2600), (12, 8192, 5000)):
        L, R, _ = synth.pair(seed, nL, nR)
        dL = torch.from_numpy(L).to(dev)
        dR = torch.from_numpy(R).to(dev)
        dPairs = torch.full((min(nL, nR), 2), -7, dtype=torch.int32, device=dev)
        dCount = torch.full((1,), -7, dtype=torch.int32, device=dev)
        st = fn(0, dL.data_ptr(), nL, dR.data_ptr(), nR, 0.7, 0.8, dPairs.data_ptr(), dCount.data_ptr(),
                C.c_void_p(stream.cuda_stream))
        assert st == v3dm_mod.OK
        torch.cuda.synchronize(dev)
        n = int(dCount.item())
        got = dPairs[:n].cpu().numpy() if n > 0 else np.zeros((0, 2), np.int32)
        with v3dm_mod.SIFTMatching(0) as m:
            m.allocate(nL, nR)
            m.set_left_features(L)
            m.set_right_features(R)
            exp = m.find_putative_matches(0.7, 0.8)
        assert n == exp.shape[0] and n > 100
        np.testing.assert_array_equal(got, exp)


def test_noalloc_rejects_sizes_above_its_limit(v3dm_mod):
    fn = _entry(v3dm_mod)
    big = v3dm_mod.lib()  # keep the library loaded
    assert big is not None
    st = fn(0, C.c_void_p(16), 8193, C.c_void_p(16), 10, 0.7, 0.8, C.c_void_p(16), C.c_void_p(16), None)
    assert st == v3dm_mod.ERR_SIZE


def test_noalloc_reports_candidate_overflow(v3dm_mod):
    """Identical descriptors on both sides make every score a candidate: 2048 x 2048 = 4.2M
    candidates against a fixed list of 524288.  The call must report -1 pairs (writes past the
    list are skipped, not performed), and the next call on good data must still be exact."""
    import torch
    dev = torch.device("cuda", 0)
    fn = _entry(v3dm_mod)
    stream = torch.cuda.current_stream(dev)
    n = 2048
    one, _, _ = synth.pair(13, 1, 1)
    same = np.repeat(one[:1], n, axis=0)
    d = torch.from_numpy(same).to(dev)
    dPairs = torch.full((n, 2), -7, dtype=torch.int32, device=dev)
    dCount = torch.full((1,), -7, dtype=torch.int32, device=dev)
    st = fn(0, d.data_ptr(), n, d.data_ptr(), n, 0.7, 0.8, dPairs.data_ptr(), dCount.data_ptr(),
            C.c_void_p(stream.cuda_stream))
    assert st == v3dm_mod.OK
    torch.cuda.synchronize(dev)
    assert int(dCount.item()) == -1
    L, R, _ = synth.pair(14, 2000, 2100)
    dL = torch.from_numpy(L).to(dev)
    dR = torch.from_numpy(R).to(dev)
    st = fn(0, dL.data_ptr(), 2000, dR.data_ptr(), 2100, 0.7, 0.8, dPairs.data_ptr(), dCount.data_ptr(),
            C.c_void_p(stream.cuda_stream))
    assert st == v3dm_mod.OK
    torch.cuda.synchronize(dev)
    k = int(dCount.item())
    with v3dm_mod.SIFTMatching(0) as m:
        m.allocate(2000, 2100)
        m.set_left_features(L)
        m.set_right_features(R)
        exp = m.find_putative_matches(0.7, 0.8)
    assert k == exp.shape[0]
    np.testing.assert_array_equal(dPairs[:k].cpu().numpy(), exp)


def test_noalloc_rejects_a_device_ordinal_past_the_device_count(v3dm_mod):
    import torch
    bad = torch.cuda.device_count()
    fn = _entry(v3dm_mod)
    st = fn(bad, C.c_void_p(16), 10, C.c_void_p(16), 10, 0.7, 0.8, C.c_void_p(16), C.c_void_p(16), None)
    assert st == v3dm_mod.ERR_ARG
