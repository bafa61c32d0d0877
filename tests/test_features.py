"""Feature-file ingestion, CPU part: the library's parser of the reference's binary feature
archive (v3dm_features_read) against the reference's own serializer
(V3D/Base/v3d_serialization.h:956-1017 over SerializableVector<SIFT_Feature>,
V3D/Base/v3d_feature.h:12-47).  The parser is host code, so these tests need no GPU."""
from pathlib import Path

import numpy as np
import pytest

from v3dm import synth

GOLDEN = Path(__file__).resolve().parent / "golden"
FIELDS = ("ids", "positions", "directions", "scales", "magnitudes", "descriptors")


def _same_bytes(a: dict, b: dict):
    for k in FIELDS:
        assert np.ascontiguousarray(a[k]).tobytes() == np.ascontiguousarray(b[k]).tobytes(), k


def test_reads_reference_written_fixture(v3dm_mod):
    """The committed archive was written by the reference's serializeDataToFile; its reader's
    arrays are committed beside it.  Byte equality, NaN and negative zero included."""
    got = v3dm_mod.features_read(GOLDEN / "features_ref.features")
    exp = np.load(GOLDEN / "features_ref.npz")
    assert got["ids"].shape[0] == 45
    _same_bytes(got, exp)


def test_matches_reference_reader_on_random_archives(v3dm_mod, oracle_mod, tmp_path):
    if not oracle_mod.ref_features_available():
        pytest.skip("reference serializer not built (oracle/_ref)")
    rng = np.random.default_rng(3)
    for n in (0, 1, 31, 2048, 2049, 5000):
        f = synth.feature_arrays(rng, n)
        f["descriptors"] = rng.standard_normal((n, 128)).astype(np.float32)
        p = tmp_path / f"r{n}.features"
        oracle_mod.ref_features_write(p, f)
        got = v3dm_mod.features_read(p)
        _same_bytes(got, oracle_mod.ref_features_read(p))
        _same_bytes(got, f)


def test_python_writer_equals_reference_writer(oracle_mod, tmp_path):
    """synth.write_features (used to make the bench's files) writes the reference's bytes."""
    if not oracle_mod.ref_features_available():
        pytest.skip("reference serializer not built (oracle/_ref)")
    f = synth.feature_arrays(np.random.default_rng(4), 300)
    a, b = tmp_path / "a.features", tmp_path / "b.features"
    synth.write_features(a, f)
    oracle_mod.ref_features_write(b, f)
    assert a.read_bytes() == b.read_bytes()


def test_errors_and_count_query(v3dm_mod, tmp_path):
    import ctypes as C
    L = v3dm_mod.lib()
    f = synth.feature_arrays(np.random.default_rng(5), 10)
    good = tmp_path / "g.features"
    synth.write_features(good, f)
    n = C.c_int32(-1)
    # count only
    assert L.v3dm_features_read(str(good).encode(), 0, C.byref(n), *([None] * 6)) == v3dm_mod.OK
    assert n.value == 10
    # too small a capacity for the arrays asked for
    ids = np.empty(10, np.int32)
    assert L.v3dm_features_read(str(good).encode(), 9, C.byref(n), ids.ctypes.data, *([None] * 5)) == \
        v3dm_mod.ERR_CAPACITY
    # only some fields
    assert L.v3dm_features_read(str(good).encode(), 10, C.byref(n), ids.ctypes.data, *([None] * 5)) == v3dm_mod.OK
    np.testing.assert_array_equal(ids, f["ids"])
    # missing file, unknown tag, text archive, truncated archive
    raw = good.read_bytes()
    bad_tag, txt, short = tmp_path / "t.features", tmp_path / "x.features", tmp_path / "s.features"
    bad_tag.write_bytes(b"V3DXXX" + raw[6:])
    txt.write_bytes(b"V3DTXT\n1\n")
    short.write_bytes(raw[:-1])
    for p, st in ((tmp_path / "missing.features", v3dm_mod.ERR_IO), (bad_tag, v3dm_mod.ERR_IO),
                  (txt, v3dm_mod.ERR_UNSUPPORTED), (short, v3dm_mod.ERR_IO)):
        assert L.v3dm_features_read(str(p).encode(), 0, C.byref(n), *([None] * 6)) == st, p.name
        with pytest.raises(v3dm_mod.V3DMError) as e:
            v3dm_mod.features_read(p)
        assert e.value.status == st
