"""The C++ compat header (the reference's V3D_CUDA class surface) compiles, links and matches
the oracle, including the reference's rounding of feature counts to multiples of 32
(V3D/CUDA/v3d_cudamatching.cu:444-519) and traverseTree's clamping (.cu:791-797)."""
import shutil
import struct
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT
from v3dm import synth

SRC = ROOT / "tests" / "compat_main.cpp"


@pytest.fixture(scope="module")
def compat_bin(tmp_path_factory, v3dm_mod):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("compat") / "compat_main"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(PKG / "compat"), "-I", str(ROOT / "include"),
           str(SRC), "-o", str(out), "-L", str(PKG), "-lv3dm", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def _run(bin_path, mode, payload, tmp_path):
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    fin.write_bytes(payload)
    p = subprocess.run([str(bin_path), mode, str(fin), str(fout)], capture_output=True, text=True, timeout=600)
    return p, fout


def _match_payload(L, R, lp, rp, F, min_score, min_ratio, thr):
    head = struct.pack("<iifff", L.shape[0], R.shape[0], min_score, min_ratio, thr)
    return b"".join([head, np.asarray(F, np.float64).tobytes(), (L.astype(np.float32) / 512).tobytes(),
                     (R.astype(np.float32) / 512).tobytes(), lp.astype(np.float32).tobytes(),
                     rp.astype(np.float32).tobytes()])


def _read_pairs(buf, off):
    n = struct.unpack_from("<i", buf, off)[0]
    pairs = np.frombuffer(buf, np.int32, 2 * n, off + 4).reshape(n, 2)
    return pairs, off + 4 + 8 * n


def test_header_compiles_and_links(compat_bin):
    assert compat_bin.exists()


def test_fails_loudly_without_gpu(compat_bin, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L, R, lp, rp, F, _ = synth.stereo(5, 64, 64)
    p, _ = _run(compat_bin, "match", _match_payload(L, R, lp, rp, F, 0.7, 0.8, 2.0), tmp_path)
    assert p.returncode == 1
    assert "V3D_CUDA SIFT_Matching(): no sm_100 CUDA device" in p.stderr


@pytest.mark.gpu
def test_match_sequence_calls(compat_bin, oracle_mod, tmp_path):
    """1000 x 1037 features: the header rounds both down (992, 1024) as the reference does."""
    L, R, lp, rp, F, _ = synth.stereo(11, 1000, 1037)
    p, fout = _run(compat_bin, "match", _match_payload(L, R, lp, rp, F, 0.7, 0.8, 2.0), tmp_path)
    assert p.returncode == 0, p.stderr
    buf = fout.read_bytes()
    put, off = _read_pairs(buf, 0)
    gui, off = _read_pairs(buf, off)
    assert off == len(buf)
    nl, nr = 992, 1024
    np.testing.assert_array_equal(put, oracle_mod.match(L[:nl], R[:nr], 0.7, 0.8))
    exp = oracle_mod.match(L[:nl], R[:nr], 0.7, 0.8, gates=[("F", F, 2.0)], lpos=lp[:nl], rpos=rp[:nr])
    np.testing.assert_array_equal(gui, exp)
    assert put.shape[0] > 100 and gui.shape[0] > 100


@pytest.mark.gpu
def test_match_using_voctree_calls(compat_bin, v3dm_mod, oracle_mod, tmp_path):
    """VocabularyTreeTraversal<10, 3>: 1000 keys, allocate rounds to 992, traverseTree clamps."""
    rng = synth.rng_for(21)
    nodes = synth.sift_like(rng, v3dm_mod.voctree_counts(10, 3)[0])
    keys = synth.sift_like(rng, 1000)
    payload = b"".join([struct.pack("<i", 1000), (nodes.astype(np.float32) / 512).tobytes(),
                        (keys.astype(np.float32) / 512).tobytes()])
    p, fout = _run(compat_bin, "voctree", payload, tmp_path)
    assert p.returncode == 0, p.stderr
    assert "Reducing nFeatures" in p.stderr
    ids = np.frombuffer(fout.read_bytes(), np.int32)
    np.testing.assert_array_equal(ids[:992], oracle_mod.voctree(10, 3, nodes, keys[:992], True))
    assert np.all(ids[992:] == -1)


@pytest.fixture(scope="module")
def stages_bin(tmp_path_factory, v3dm_mod):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("stages") / "compat_stages"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(PKG / "compat"), "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "compat_stages.cpp"), "-o", str(out), "-L", str(PKG), "-lv3dm", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def test_stages_header_compiles_and_links(stages_bin):
    """compat/V3DM/v3dm_sfm_stages.h (retrieval loop and robust orientation of many pairs) with the
    apps' member names."""
    assert stages_bin.exists()


@pytest.mark.parametrize("mode,who", [("r", "computeRobustOrientationBatch()"), ("w", "retrieveSequence()")])
def test_stages_fail_loudly_without_gpu(stages_bin, mode, who):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = subprocess.run([str(stages_bin), mode], capture_output=True, text=True, timeout=120)
    assert p.returncode == 1
    assert f"V3D_B200 {who}: no sm_100" in p.stderr


def _views_payload(views, pairs, F, thr, n_max, min_score, min_ratio):
    """views: list of (positions (n, 2), float descriptors (n, 128)); pairs (view1, view2)."""
    parts = [struct.pack("<iiiff", len(views), len(pairs), n_max, min_score, min_ratio)]
    for pos, desc in views:
        parts.append(struct.pack("<i", desc.shape[0]))
        rec = np.concatenate([np.asarray(pos, np.float32), np.asarray(desc, np.float32)], axis=1)
        parts.append(np.ascontiguousarray(rec, np.float32).tobytes())
    for k, (a, b) in enumerate(pairs):
        parts.append(struct.pack("<ii", int(a), int(b)))
        parts.append(np.asarray(F[k], np.float64).tobytes())
        parts.append(struct.pack("<f", float(thr[k])))
    return b"".join(parts)


def _read_matches(buf, n_pairs):
    out, off = [], 0
    for _ in range(n_pairs):
        pr, off = _read_pairs(buf, off)
        out.append(pr)
    assert off == len(buf)
    return out


@pytest.mark.parametrize("mode,who", [("m", "findPutativeMatchesBatch()"), ("g", "runGuidedMatchingBatch()")])
def test_matching_stages_fail_loudly_without_gpu(stages_bin, mode, who, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rng = np.random.default_rng(0)
    views = [(rng.uniform(0, 100, (40, 2)), rng.uniform(0, 1, (40, 128))) for _ in range(2)]
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    fin.write_bytes(_views_payload(views, [(0, 1)], [np.eye(3)], [2.0], 4096, 0.7, 0.8))
    p = subprocess.run([str(stages_bin), mode, str(fin), str(fout)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 1
    assert f"V3D_B200 {who}: no sm_100" in p.stderr


@pytest.mark.gpu
def test_matching_stages_equal_the_app_loop(stages_bin, oracle_mod, v3dm_mod, tmp_path):
    """The app's per-pair loop (match_sequence.cpp:165-234, :306-324) with its count rounding
    (min(nMaxFeatures, size & 0xffe0)): u/512 views against the oracle (putative and F-guided),
    float views against the single-pair float matcher."""
    desc8, counts, offs, pos, cams = synth.scene(24, 5, 300, 1500)
    n_max = 1200
    cut = [min(n_max, int(c) & 0xffe0) for c in counts]
    pairs = [(0, 1), (1, 2), (0, 2), (3, 4), (2, 4), (4, 0)]
    F = [synth.fundamental(cams, a, b) for a, b in pairs]
    thr = [2.0, 8.0, 2.0, 2.0, 8.0, 2.0]
    views8 = [(pos[offs[v]:offs[v + 1]], desc8[offs[v]:offs[v + 1]].astype(np.float32) / 512) for v in range(5)]
    for mode in ("m", "g"):
        fin, fout = tmp_path / f"in_{mode}.bin", tmp_path / f"out_{mode}.bin"
        fin.write_bytes(_views_payload(views8, pairs, F, thr, n_max, 0.7, 0.8))
        p = subprocess.run([str(stages_bin), mode, str(fin), str(fout)], capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        got = _read_matches(fout.read_bytes(), len(pairs))
        for k, (a, b) in enumerate(pairs):
            L = desc8[offs[a]:offs[a] + cut[a]]
            R = desc8[offs[b]:offs[b] + cut[b]]
            if mode == "m":
                exp = oracle_mod.match(L, R, 0.7, 0.8)
            else:
                exp = oracle_mod.match(L, R, 0.7, 0.8, gates=[("F", F[k], thr[k])], lpos=pos[offs[a]:offs[a] + cut[a]],
                                       rpos=pos[offs[b]:offs[b] + cut[b]])
            np.testing.assert_array_equal(got[k], exp, err_msg=f"{mode} pair {k}")
    # float descriptors (not u/512): the single-pair float matcher's putative result
    descf = synth.float_from_u8(desc8, 24)
    viewsf = [(pos[offs[v]:offs[v + 1]], descf[offs[v]:offs[v + 1]]) for v in range(5)]
    fin, fout = tmp_path / "in_f.bin", tmp_path / "out_f.bin"
    fin.write_bytes(_views_payload(viewsf, pairs, F, thr, n_max, 0.7, 0.8))
    p = subprocess.run([str(stages_bin), "m", str(fin), str(fout)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    got = _read_matches(fout.read_bytes(), len(pairs))
    for k, (a, b) in enumerate(pairs):
        with v3dm_mod.SIFTMatching(0) as m:
            m.allocate(cut[a], cut[b], False)
            m.set_left_features(descf[offs[a]:offs[a] + cut[a]])
            m.set_right_features(descf[offs[b]:offs[b] + cut[b]])
            np.testing.assert_array_equal(got[k], m.find_putative_matches(0.7, 0.8), err_msg=f"float pair {k}")
