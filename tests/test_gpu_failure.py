"""Failure path of the tensor-core side pass, exercised without faulting the GPU.

Every device wait of the side kernel is bounded.  The matcher's test hook makes CTA 0's producer
leave one B tile unloaded and shortens the waits, so the MMA issuer's wait for that tile runs
out: the CTA aborts (every role stops, waits for its own copies and MMAs in flight, frees TMEM),
the other CTAs finish, and the call reports V3DM_ERR_TIMEOUT.  The handle must stay usable: with
the hook off, the next calls give the oracle's pairs.  The reference has no such path: it prints
and exits on any CUDA error (v3d_cudamatching.cu:12-27)."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


def test_a_wait_that_runs_out_reports_timeout_and_the_handle_recovers(v3dm_mod, oracle_mod):
    # 6000 x 5600 with 128 x 256 tiles: 47 x 22 tiles over 148 CTAs, so CTA 0 loads six B tiles
    L, R, lp, rp, F, _ = synth.stereo(23, 6000, 5600)
    exp = oracle_mod.match(L, R, 0.7, 0.8)
    exp_g = oracle_mod.match(L, R, 0.7, 0.8, gates=[("F", F, 2.0)], lpos=lp, rpos=rp)
    with v3dm_mod.SIFTMatching(0) as m:
        m.allocate(6000, 5600, True)
        m.set_config(0)
        m.set_left_features(L)
        m.set_right_features(R)
        np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), exp)
        for skip in (1, 3):
            m.test_wait_fault(20_000_000, skip)  # ~10 ms at the B200's clocks
            m.profile(True)
            status = v3dm_mod.OK
            try:
                m.find_putative_matches(0.7, 0.8)
            except v3dm_mod.V3DMError as e:
                status = e.status
            pass_a_ms, _ = m.profile_read(0)
            m.profile(False)
            print(f"skip {skip}: status {status}, pass A {pass_a_ms:.3f} ms")
            assert status == v3dm_mod.ERR_TIMEOUT, (status, pass_a_ms)
            assert pass_a_ms >= 5.0  # the pass lasted as long as the shortened wait
            # a guided call after the failed pass recomputes it (the cached pass is incomplete)
            m.test_wait_fault(0, 0)
            np.testing.assert_array_equal(m.run_guided_matching(F, 2.0, lp, rp, 0.7, 0.8), exp_g)
            np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), exp)


def test_short_wait_limit_alone_does_not_fail_a_call(v3dm_mod, oracle_mod):
    """A wait limit well above a tile's latency, with every load issued, changes nothing."""
    L, R, _ = synth.pair(24, 2000, 2100)
    with v3dm_mod.SIFTMatching(0) as m:
        m.allocate(2000, 2100)
        m.set_left_features(L)
        m.set_right_features(R)
        m.test_wait_fault(200_000_000, 0)
        np.testing.assert_array_equal(m.find_putative_matches(0.7, 0.8), oracle_mod.match(L, R, 0.7, 0.8))
        m.test_wait_fault(0, 0)


def test_hook_arguments(v3dm_mod):
    with v3dm_mod.SIFTMatching(0) as m:
        for args in ((-1, 0), (10, -1), (0, 2)):
            with pytest.raises(v3dm_mod.V3DMError) as e:
                m.test_wait_fault(*args)
            assert e.value.status == v3dm_mod.ERR_ARG
