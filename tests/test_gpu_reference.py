"""Pins the oracle to the reference itself: the reference's own CUDA matcher
(V3D/CUDA/v3d_cudamatching.cu, built unmodified with CUDA 12.9 through oracle/ref_cuda_shim.h
into oracle/_ref/libv3dref_cuda.so) run on the GPU, against the oracle on the same inputs.

The reference's build uses --use_fast_math, so its divisions are approximate; on uint8
descriptors the ratio decision is nevertheless exact (see the oracle's header), and the
cases below are required to agree bit for bit."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_available(oracle_mod):
    if not oracle_mod.ref_cuda_available():
        pytest.fail("oracle/_ref/libv3dref_cuda.so is missing; build it with `make -C oracle ref` where the "
                    "reference sources are present")
    return True


@pytest.mark.parametrize("seed,n", [(0, 1024), (1, 4096), (2, 2048)])
@pytest.mark.parametrize("ms,mr", [(0.7, 0.8), (0.9, 0.8), (0.7, -1.0)])
def test_reference_putative_equals_oracle(ref_available, oracle_mod, tmp_path, seed, n, ms, mr):
    L, R, _ = synth.pair(seed, n, n)
    exp = oracle_mod.match(L, R, ms, mr)
    got = oracle_mod.ref_cuda_match(L, R, ms, mr, workdir=str(tmp_path))
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("seed", [1, 2])
def test_reference_guided_equals_oracle(ref_available, oracle_mod, tmp_path, seed):
    L, R, lp, rp, F, _ = synth.stereo(seed, 2048, 2048)
    H = np.array([[1.0, 0.01, 25.0], [0.0, 1.0, 3.0], [0.0, 0.0, 1.0]])
    for gates in ([("F", F, 2.0)], [("H", H, 300.0)], [("F", F, 4.0), ("H", H, 600.0)]):
        exp = oracle_mod.match(L, R, 0.7, 0.8, gates=gates, lpos=lp, rpos=rp)
        got = oracle_mod.ref_cuda_match(L, R, 0.7, 0.8, gates=gates, lpos=lp, rpos=rp, workdir=str(tmp_path))
        np.testing.assert_array_equal(got, exp)
