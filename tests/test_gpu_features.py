"""Feature-file ingestion on the GPU: the loader (v3dm_loader_*) and the u8 re-quantisation
kernel (v3dm_quantize_u8_device), checked against the reference's reader (through the library's
host parser, pinned to it by tests/test_features.py) and a numpy statement of the quantisation;
then the loaded descriptors feed the matchers and give the host path's results."""
import numpy as np
import pytest

from v3dm import synth

pytestmark = pytest.mark.gpu


def _quantize(x):
    """u = round(512 x), half to even, clamped to 0..255; NaN -> 0."""
    q = np.rint(np.nan_to_num(x.astype(np.float32), nan=0.0, posinf=np.inf, neginf=-np.inf) * np.float32(512))
    return np.clip(q, 0, 255).astype(np.uint8)


def test_quantize_kernel_edges(v3dm_mod):
    import torch
    vals = np.array([0.0, -0.0, 0.5 / 512, 1.5 / 512, 2.5 / 512, 255.49 / 512, 255.5 / 512, 300.0, -1.0, np.nan,
                     np.inf, -np.inf, 1e-45, 17.0 / 512, 0.49999997 / 512, 254.5 / 512], np.float32)
    x = np.concatenate([vals, np.random.default_rng(1).uniform(-0.1, 0.6, 4096 - vals.size).astype(np.float32)])
    d = torch.from_numpy(x).cuda()
    out = torch.empty(x.size, dtype=torch.uint8, device="cuda")
    v3dm_mod.quantize_u8_device(d.data_ptr(), x.size, out.data_ptr(), 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), _quantize(x))
    # u/512 inputs come back unchanged
    u = np.arange(256, dtype=np.uint8)
    d2 = torch.from_numpy(u.astype(np.float32) / 512).cuda()
    out2 = torch.empty(256, dtype=torch.uint8, device="cuda")
    v3dm_mod.quantize_u8_device(d2.data_ptr(), 256, out2.data_ptr(), 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out2.cpu().numpy(), u)


def _device_bytes(ptr, nbytes):
    """A host copy of nbytes of device memory at ptr (a torch view through the CUDA array
    interface)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}

    if nbytes == 0:
        return np.zeros(0, np.uint8)
    return torch.as_tensor(_View(), device="cuda").cpu().numpy()


def _files(tmp_path, counts, seed=2, real_floats=False, text=()):
    """Feature files; those whose index is in text are text archives (V3DTXT) laid out as the
    reference's text serializer writes them."""
    rng = np.random.default_rng(seed)
    paths, feats = [], []
    for i, n in enumerate(counts):
        f = synth.feature_arrays(rng, n)
        if real_floats:  # unit-norm float descriptors, not of the form u/512
            x = rng.gamma(0.6, 1.0, (n, 128)).astype(np.float32)
            f["descriptors"] = (x / np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)).astype(np.float32)
        p = tmp_path / f"img{i}.features"
        if i in text:
            synth.write_features_text(p, f)
        else:
            synth.write_features(p, f)
        paths.append(str(p))
        feats.append(f)
    return paths, feats


@pytest.mark.parametrize("max_per_image,flags", [(0, 0), (0, 1), (700, 0), (700, 1)])
def test_loader_equals_reader_and_quantisation(v3dm_mod, tmp_path, max_per_image, flags):
    """Unit-L2 float files rounded on request (LOAD_LOSSY_U8) equal the reader's floats
    quantised by numpy; the positions equal the reader's."""
    counts = [1000, 0, 31, 33, 2500, 700, 64]
    paths, feats = _files(tmp_path, counts, real_floats=True, text=(2, 4))
    flags |= v3dm_mod.LOAD_LOSSY_U8
    with v3dm_mod.Loader() as ld:
        kept = ld.load(paths, max_per_image, flags)
        assert not ld.exact_u8()
        exp_kept = []
        for n in counts:
            k = n & ~31 if flags & v3dm_mod.LOAD_ROUND32 else n
            exp_kept.append(min(k, max_per_image) if max_per_image > 0 else k)
        np.testing.assert_array_equal(kept, exp_kept)
        d_ptr, total = ld.descriptors_device()
        assert total == sum(exp_kept)
        got = _device_bytes(d_ptr, total * 128).reshape(total, 128)
        pos = ld.positions()
    exp_desc = np.concatenate([v3dm_mod.features_read(p)["descriptors"][:k] for p, k in zip(paths, exp_kept)])
    exp_pos = np.concatenate([v3dm_mod.features_read(p)["positions"][:k] for p, k in zip(paths, exp_kept)])
    np.testing.assert_array_equal(got, _quantize(exp_desc))
    np.testing.assert_array_equal(pos, exp_pos)


def test_loaded_descriptors_feed_the_matchers(v3dm_mod, tmp_path):
    """Batched all-pairs matching of loaded files equals matching of the same descriptors
    quantised on the host; a single pair set from the loader's device buffer likewise."""
    desc, counts, offs = synth.images(31, n_images=6, n_min=800, n_max=3000)
    rng = np.random.default_rng(6)
    paths = []
    for i in range(6):
        f = synth.feature_arrays(rng, int(counts[i]), desc[offs[i]:offs[i + 1]])
        p = tmp_path / f"v{i}.features"
        synth.write_features(p, f)
        paths.append(str(p))
    with v3dm_mod.Loader() as ld:
        kept = ld.load(paths)
        np.testing.assert_array_equal(kept, counts)
        d_ptr, total = ld.descriptors_device()
        b = v3dm_mod.BatchMatching()
        b.set_images_device(d_ptr, kept)
        b.set_pairs(None)
        got = b.match(0.7, 0.8)
        b2 = v3dm_mod.BatchMatching()
        b2.set_images(desc, counts)
        b2.set_pairs(None)
        np.testing.assert_array_equal(got, b2.match(0.7, 0.8))
        assert got.shape[0] > 0
        b.close()
        b2.close()
        m = v3dm_mod.SIFTMatching()
        m.allocate(3000, 3000)
        m.set_left_features_device(d_ptr + int(offs[0]) * 128, int(counts[0]))
        m.set_right_features_device(d_ptr + int(offs[3]) * 128, int(counts[3]))
        a = m.find_putative_matches(0.7, 0.8)
        m.set_left_features(desc[offs[0]:offs[1]])
        m.set_right_features(desc[offs[3]:offs[4]])
        np.testing.assert_array_equal(a, m.find_putative_matches(0.7, 0.8))
        m.close()


def test_loader_errors(v3dm_mod, tmp_path):
    paths, _ = _files(tmp_path, [100, 50])
    (tmp_path / "bad.features").write_bytes(b"V3DTXT\n1\n")
    with v3dm_mod.Loader() as ld:
        with pytest.raises(v3dm_mod.V3DMError) as e:
            ld.load(paths + [str(tmp_path / "missing.features")])
        assert e.value.status == v3dm_mod.ERR_IO
        with pytest.raises(v3dm_mod.V3DMError) as e:  # a text archive without its brackets
            ld.load([str(tmp_path / "bad.features")])
        assert e.value.status == v3dm_mod.ERR_IO
        # still usable after an error
        np.testing.assert_array_equal(ld.load(paths), [100, 50])


def test_loader_refuses_to_round_unit_floats_silently(v3dm_mod, tmp_path):
    """The extractors store unit-L2 floats; without LOAD_LOSSY_U8 or LOAD_KEEP_F32 the loader
    reports them instead of rounding them.  u/512 files load as u8 with no flag."""
    paths, _ = _files(tmp_path, [300, 200], real_floats=True)
    (tmp_path / "u").mkdir()
    upaths, ufeats = _files(tmp_path / "u", [300, 200])
    with v3dm_mod.Loader() as ld:
        with pytest.raises(v3dm_mod.V3DMError) as e:
            ld.load(paths)
        assert e.value.status == v3dm_mod.ERR_NOT_U8
        np.testing.assert_array_equal(ld.load(upaths), [300, 200])
        assert ld.exact_u8()
        d_ptr, total = ld.descriptors_device()
        got = _device_bytes(d_ptr, total * 128).reshape(total, 128)
        np.testing.assert_array_equal(got, np.concatenate([_quantize(f["descriptors"]) for f in ufeats]))
        # floats kept: the u8 view is refused, the float view is the file's floats
        ld.load(paths, 0, v3dm_mod.LOAD_KEEP_F32)
        with pytest.raises(v3dm_mod.V3DMError) as e:
            ld.descriptors_device()
        assert e.value.status == v3dm_mod.ERR_NOT_U8


def _device_floats(ptr, n):
    raw = _device_bytes(ptr, n * 4)
    return raw.view(np.float32)


def test_loader_keeps_floats_for_the_float_matcher(v3dm_mod, tmp_path):
    """Feature files of unit-L2 float descriptors (what the extractors write): the loader keeps
    the floats bit for bit (LOAD_KEEP_F32), and matching them from the loader's device buffer
    gives the same pairs as matching the in-memory floats (the BF16 hi/lo path), for putative
    and F-guided matching."""
    L, R, lp, rp, F, _ = synth.stereo(17, 1800, 2100)
    rng = np.random.default_rng(3)
    # unit-L2 floats with the generator's directions (not u/512)
    Lf = (L.astype(np.float32) + rng.uniform(-0.49, 0.49, L.shape).astype(np.float32))
    Rf = (R.astype(np.float32) + rng.uniform(-0.49, 0.49, R.shape).astype(np.float32))
    Lf = np.maximum(Lf, 0) / np.linalg.norm(np.maximum(Lf, 0), axis=1, keepdims=True)
    Rf = np.maximum(Rf, 0) / np.linalg.norm(np.maximum(Rf, 0), axis=1, keepdims=True)
    Lf, Rf = Lf.astype(np.float32), Rf.astype(np.float32)
    paths = []
    for i, (D, P) in enumerate(((Lf, lp), (Rf, rp))):
        f = synth.feature_arrays(rng, D.shape[0])
        f["descriptors"] = D
        f["positions"] = P.astype(np.float32)
        path = tmp_path / f"s{i}.features"
        synth.write_features(path, f)
        paths.append(str(path))
    with v3dm_mod.Loader() as ld:
        kept = ld.load(paths, 0, v3dm_mod.LOAD_KEEP_F32)
        np.testing.assert_array_equal(kept, [1800, 2100])
        assert not ld.exact_u8()
        d_ptr, total = ld.descriptors_f32_device()
        assert total == 3900
        np.testing.assert_array_equal(_device_floats(d_ptr, total * 128).reshape(total, 128),
                                      np.concatenate([Lf, Rf]))
        pos = ld.positions()
        np.testing.assert_array_equal(pos, np.concatenate([lp, rp]).astype(np.float32))
        with v3dm_mod.SIFTMatching() as m:
            m.allocate(2100, 2100, True)
            m.set_left_features_f32_device(d_ptr, 1800)
            m.set_right_features_f32_device(d_ptr + 1800 * 128 * 4, 2100)
            put = m.find_putative_matches(0.7, 0.8)
            gui = m.run_guided_matching(F, 2.0, pos[:1800], pos[1800:], 0.7, 0.8)
            m.set_left_features(Lf)
            m.set_right_features(Rf)
            np.testing.assert_array_equal(put, m.find_putative_matches(0.7, 0.8))
            np.testing.assert_array_equal(gui, m.run_guided_matching(F, 2.0, lp, rp, 0.7, 0.8))
            assert put.shape[0] > 100 and 0 < gui.shape[0] <= put.shape[0]
