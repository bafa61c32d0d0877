"""CPU checks of the inputs the float workloads and the bench lines are built from: the float
descriptors of the batched float tests and of `bench.py --workload batch-float` (unit length, not
of the form u/512 so that they take the BF16 hi/lo path, close to their uint8 source so that the
shared tracks still match), and the peak denominators of the roofline fields."""
import json
import sys
from pathlib import Path

import numpy as np

from v3dm import synth

ROOT = Path(__file__).resolve().parents[1]


def test_float_from_u8_is_unit_length_and_not_u512():
    desc, counts, offs = synth.images(3, 4, 200, 400)
    f = synth.float_from_u8(desc, 3)
    assert f.dtype == np.float32 and f.shape == desc.shape
    np.testing.assert_allclose(np.linalg.norm(f.astype(np.float64), axis=1), 1.0, atol=1e-5)
    assert (f >= 0).all()
    u = f * 512
    assert np.abs(u - np.rint(u)).max() > 1e-3  # not u/512: the float path, not the integer one
    # the same seed gives the same descriptors; the perturbation keeps them near their source
    np.testing.assert_array_equal(f, synth.float_from_u8(desc, 3))
    src = desc.astype(np.float64) / 512
    src /= np.linalg.norm(src, axis=1, keepdims=True)
    cos = np.einsum("ij,ij->i", src, f.astype(np.float64))
    assert cos.min() > 0.98


def test_sustained_fraction_fields():
    sys.path.insert(0, str(ROOT))
    import bench
    peaks = {"bf16_tflops": 1600.0, "bf16_tflops_sustained": 1400.0}
    d = bench.sustained_fields(1400.0, peaks, 2.0)
    assert d == {"peak_sustained": 2800.0, "frac_sustained": 0.5}
    assert bench.sustained_fields(1.0, {"bf16_tflops": 1.0}, 1.0) == {}


def test_load_peaks_reads_the_measured_file():
    sys.path.insert(0, str(ROOT))
    import bench
    p = bench.load_peaks()
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        assert p["src"] == "measured"
        assert p["bf16_tflops"] == d["bf16_tflops"] and p["hbm_gbs"] == d["hbm_gbs"]
        assert p["bf16_tflops_sustained"] == d.get("bf16_tflops_sustained")
    else:
        assert p["src"] == "fallback"
