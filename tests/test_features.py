"""Feature-file ingestion, CPU part: the library's parser of the reference's binary and text
feature archives (v3dm_features_read) against the reference's own serializer
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


def test_reads_reference_written_text_fixture(v3dm_mod):
    """A text archive written by the reference (writeBinary = false) and what the reference's
    reader returns for it: the parser rounds the printed decimals as the stream extraction does
    (extreme ids, negative zero, a denormal, the largest float, float minimum normal)."""
    got = v3dm_mod.features_read(GOLDEN / "features_ref_text.features")
    exp = np.load(GOLDEN / "features_ref_text.npz")
    assert got["ids"].shape[0] == 23
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
        t = tmp_path / f"r{n}.txt.features"
        oracle_mod.ref_features_write(t, f, binary=False)
        _same_bytes(v3dm_mod.features_read(t), oracle_mod.ref_features_read(t))


def test_python_writer_equals_reference_writer(oracle_mod, tmp_path):
    """synth.write_features (used to make the bench's files) writes the reference's bytes."""
    if not oracle_mod.ref_features_available():
        pytest.skip("reference serializer not built (oracle/_ref)")
    f = synth.feature_arrays(np.random.default_rng(4), 300)
    a, b = tmp_path / "a.features", tmp_path / "b.features"
    synth.write_features(a, f)
    oracle_mod.ref_features_write(b, f)
    assert a.read_bytes() == b.read_bytes()


def test_python_text_writer_equals_reference_text_writer(oracle_mod, tmp_path):
    if not oracle_mod.ref_features_available():
        pytest.skip("reference serializer not built (oracle/_ref)")
    for n in (0, 1, 40):
        f = synth.feature_arrays(np.random.default_rng(7 + n), n)
        if n:
            f["descriptors"][0, :4] = np.array([-0.0, 1e-45, 1e30, 3.4028235e38], np.float32)
        a, b = tmp_path / f"a{n}.features", tmp_path / f"b{n}.features"
        synth.write_features_text(a, f)
        oracle_mod.ref_features_write(b, f, binary=False)
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
    # missing file, unknown tag, truncated archive
    raw = good.read_bytes()
    bad_tag, short = tmp_path / "t.features", tmp_path / "s.features"
    bad_tag.write_bytes(b"V3DXXX" + raw[6:])
    short.write_bytes(raw[:-1])
    for p, st in ((tmp_path / "missing.features", v3dm_mod.ERR_IO), (bad_tag, v3dm_mod.ERR_IO),
                  (short, v3dm_mod.ERR_IO)):
        assert L.v3dm_features_read(str(p).encode(), 0, C.byref(n), *([None] * 6)) == st, p.name
        with pytest.raises(v3dm_mod.V3DMError) as e:
            v3dm_mod.features_read(p)
        assert e.value.status == st


def test_text_archive_layout_and_errors(v3dm_mod, tmp_path):
    """The parser reads an archive laid out by hand the way the writer lays it out; a value the
    stream extraction cannot read (nan, inf, an overflow, a stray character), a wrong tag, a
    missing bracket or a short file gives ERR_IO (the reference throws there)."""
    f = synth.feature_arrays(np.random.default_rng(6), 4)
    p = tmp_path / "h.features"
    synth.write_features_text(p, f)
    text = p.read_text()
    got = v3dm_mod.features_read(p)
    np.testing.assert_array_equal(got["ids"], f["ids"])
    for k in ("positions", "directions", "scales", "magnitudes", "descriptors"):
        exp = np.array([np.float32(float(f"{float(v):g}")) for v in np.ravel(f[k])], np.float32)
        assert got[k].ravel().tobytes() == exp.tobytes(), k
    first = f"{float(f['descriptors'][0, 0]):g}"
    assert first in text
    bad = {
        "nan": text.replace(" " + first + " ", " nan ", 1),
        "inf": text.replace(" " + first + " ", " inf ", 1),
        "overflow": text.replace(" " + first + " ", " 1e39 ", 1),
        "stray": text.replace(" " + first + " ", " " + first + "x ", 1),
        "hex": text.replace(" " + first + " ", " 0x1p3 ", 1),
        "tag": text.replace("SIFT_Feature", "SIFT_Featurex", 1),
        "bracket": text.rstrip().rstrip("}"),
        "short": text[: len(text) // 2],
        "id_range": text.replace(f"{{ {int(f['ids'][0])} ", "{ 2147483648 ", 1),
    }
    for name, t in bad.items():
        q = tmp_path / f"bad_{name}.features"
        q.write_text(t)
        with pytest.raises(v3dm_mod.V3DMError) as e:
            v3dm_mod.features_read(q)
        assert e.value.status == v3dm_mod.ERR_IO, name
    # the count alone is read from the head of the archive
    import ctypes as C
    n = C.c_int32(-1)
    q = tmp_path / "head.features"
    q.write_text("V3DTXT\n7 { ")
    assert v3dm_mod.lib().v3dm_features_read(str(q).encode(), 0, C.byref(n), *([None] * 6)) == v3dm_mod.OK
    assert n.value == 7
