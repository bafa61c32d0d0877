"""Writes the golden fixtures of tests/golden/ from the reference's own code.

    python tests/golden/make_golden.py voctree [outdir]   # CPU: V3D::VocabularyTree::getVisualWord
    python tests/golden/make_golden.py match [outdir]     # GPU: V3D_CUDA::SIFT_Matching
    python tests/golden/make_golden.py features [outdir]  # CPU: V3D::serializeDataToFile / FromFile
    python tests/golden/make_golden.py retrieval [outdir] # CPU: V3D::LeafDocuments binomial scores
    python tests/golden/make_golden.py ransac [outdir]    # CPU: five-point solver, robust orientation loop

voctree: the reference's CPU vocabulary tree (V3D/Base/v3d_vocabularytree.h, built from the
reference headers into oracle/_ref/libv3dref_voctree.so by `make -C oracle ref`), leaf-local
ids, for every tree shape the wrapper instantiates that is small enough to store.
match: the reference's CUDA matcher (V3D/CUDA/v3d_cudamatching.cu, built unmodified into
oracle/_ref/libv3dref_cuda.so) on an sm_100 GPU: putative matching with and without the ratio
test, guided F matching and compounding F + H gates, and a case with duplicated descriptors.

features: a binary feature archive written by the reference's serializer (oracle/_ref/
libv3dref_features.so, from V3D/Base/v3d_serialization.h and v3d_feature.h) and the arrays its
reader returns for it.  The records hold edge values (negative ids, NaN, infinities, negative
zero, denormals) so that the check is on the bytes.  Beside it, a text archive ("V3DTXT") written
by the same serializer with writeBinary = false, and what its reader makes of it.

retrieval: the image loop of match_using_voctree.cpp:176-222 (computeBinomialScores, then
insertDocument) on the reference's LeafDocuments (oracle/_ref/libv3dref_retrieval.so, from
V3D/Base/v3d_voctree.h), on seeded visual-word sequences (v3dm.synth.sequence_words) and hand-made
edge cases: an empty image, identical images (equal scores, ranked by index), repeated words,
n_best above the image count, pMatch 0, a query whose every word is unseen.

ransac: the reference's computeEssentialsFromFiveCorrs on 300 normalised samples (half from a true
pose, half random), and its relativePoseFromEssential + the loop of computeRobustOrientationMLE
(oracle/_ref/libv3dref_ransac.so, from V3D/Geometry/v3d_poseutilities.cpp) on 6 synthetic pairs with
the reference's own sample draws (srand(seed), std::random_shuffle).

Inputs are SIFT-like uint8 descriptors (values u/512 handed to the reference as floats) from
v3dm.synth, stored in the fixtures together with the outputs, so the fixtures stand alone.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "eth-v3d-lgpl_b200"))
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from v3dm import synth  # noqa: E402

# (branch factor, depth, number of keys); shapes instantiated in oracle/ref_voctree_wrap.cpp
VOCTREE_CASES = [(2, 1, 100), (3, 2, 150), (4, 3, 250), (5, 4, 250), (10, 2, 250), (10, 3, 200)]

H_GATE = np.array([[1.0, 0.01, 25.0], [0.0, 1.0, 3.0], [0.0, 0.0, 1.0]])


def make_voctree(out: Path) -> None:
    if not oracle.ref_voctree_available():
        raise SystemExit("oracle/_ref/libv3dref_voctree.so missing: run `make -C oracle ref` first")
    arrays = {}
    for i, (bf, depth, n) in enumerate(VOCTREE_CASES):
        rng = synth.rng_for(1000 + i)
        n_nodes = sum(bf ** d for d in range(1, depth + 1))
        nodes = synth.sift_like(rng, n_nodes)
        keys = synth.sift_like(rng, n)
        ids = oracle.ref_voctree(bf, depth, nodes.astype(np.float32) / 512, keys.astype(np.float32) / 512)
        arrays[f"c{i}_shape"] = np.array([bf, depth], np.int32)
        arrays[f"c{i}_nodes"] = nodes
        arrays[f"c{i}_keys"] = keys
        arrays[f"c{i}_leaf_local"] = ids
    arrays["n_cases"] = np.array(len(VOCTREE_CASES), np.int32)
    np.savez_compressed(out / "voctree_ref.npz", **arrays)
    print("wrote", out / "voctree_ref.npz")


def _tie_pair():
    """Left and right sets with exact duplicates: ties in the best and second-best scores."""
    rng = synth.rng_for(77)
    base = synth.sift_like(rng, 160)
    L = np.concatenate([base[:128], base[:64], base[128:160]])  # lefts 128..191 repeat lefts 0..63
    R = np.concatenate([base[32:96], base[32:64], synth.sift_like(rng, 64), base[100:132]])
    return L.copy(), R.copy()


def make_match(out: Path) -> None:
    if not oracle.ref_cuda_available():
        raise SystemExit("oracle/_ref/libv3dref_cuda.so missing: run `make -C oracle ref` first")
    arrays = {}
    cases = []
    L, R, _ = synth.pair(10, 512, 480)
    arrays["pair_L"], arrays["pair_R"] = L, R
    for ms, mr in ((0.7, 0.8), (0.9, 0.8), (0.7, -1.0), (0.8, 0.6)):
        cases.append(("pair", ms, mr, []))
    L, R, lp, rp, F, _ = synth.stereo(12, 512, 544)
    arrays["stereo_L"], arrays["stereo_R"] = L, R
    arrays["stereo_lpos"], arrays["stereo_rpos"], arrays["stereo_F"] = lp, rp, F
    arrays["stereo_H"] = H_GATE
    cases.append(("stereo", 0.7, 0.8, []))
    cases.append(("stereo", 0.7, 0.8, [("F", 2.0)]))
    cases.append(("stereo", 0.7, -1.0, [("F", 2.0)]))
    cases.append(("stereo", 0.7, 0.8, [("H", 300.0)]))
    cases.append(("stereo", 0.7, 0.8, [("F", 4.0), ("H", 600.0)]))
    L, R = _tie_pair()
    arrays["ties_L"], arrays["ties_R"] = L, R
    for ms, mr in ((0.7, 0.8), (0.7, -1.0)):
        cases.append(("ties", ms, mr, []))
    for i, (inp, ms, mr, gates) in enumerate(cases):
        Li, Ri = arrays[f"{inp}_L"], arrays[f"{inp}_R"]
        g = [(t, arrays[f"{inp}_{t}"], thr) for t, thr in gates]
        kw = {}
        if gates:
            kw = dict(lpos=arrays[f"{inp}_lpos"], rpos=arrays[f"{inp}_rpos"])
        pairs = oracle.ref_cuda_match(Li, Ri, ms, mr, gates=g, **kw)
        arrays[f"c{i}_input"] = np.array(inp)
        arrays[f"c{i}_params"] = np.array([ms, mr], np.float32)
        arrays[f"c{i}_gates"] = np.array([f"{t}:{thr!r}" for t, thr in gates])
        arrays[f"c{i}_pairs"] = pairs.astype(np.int32)
        print(f"case {i}: {inp} ms={ms} mr={mr} gates={gates} -> {pairs.shape[0]} pairs")
    arrays["n_cases"] = np.array(len(cases), np.int32)
    np.savez_compressed(out / "match_ref.npz", **arrays)
    print("wrote", out / "match_ref.npz")


def make_features(out: Path) -> None:
    if not oracle.ref_features_available():
        raise SystemExit("oracle/_ref/libv3dref_features.so missing: run `make -C oracle ref` first")
    rng = synth.rng_for(4242)
    f = synth.feature_arrays(rng, 45)
    f["ids"][:5] = [-1, -2147483648, 2147483647, 0, 7]
    edge = np.array([np.nan, np.inf, -np.inf, -0.0, 1e-45, -3.5, 1e30, 0.5 / 512], np.float32)
    f["descriptors"][0, :edge.size] = edge
    f["positions"][1] = [np.nan, -0.0]
    f["scales"][2] = np.inf
    path = out / "features_ref.features"
    oracle.ref_features_write(path, f)
    back = oracle.ref_features_read(path)
    for k in oracle.FEATURE_FIELDS:
        assert back[k].tobytes() == np.ascontiguousarray(f[k]).tobytes(), k
    np.savez_compressed(out / "features_ref.npz", **back)
    print("wrote", path, "and", out / "features_ref.npz")
    # the text archive (writeBinary = false): values as the stream prints them (6 significant
    # digits), so the fixture holds what the reference's reader makes of that text.  Finite
    # values only: the reference cannot read back the "nan" / "inf" it prints.
    t = synth.feature_arrays(synth.rng_for(4343), 23)
    t["ids"][:3] = [-2147483648, 2147483647, 0]
    t["descriptors"][0, :8] = np.array([-0.0, 1e-45, -3.5, 1e30, 0.5 / 512, 3.4028235e38, 1.17549435e-38, 7e-39],
                                       np.float32)
    tpath = out / "features_ref_text.features"
    oracle.ref_features_write(tpath, t, binary=False)
    tback = oracle.ref_features_read(tpath)
    np.savez_compressed(out / "features_ref_text.npz", **tback)
    print("wrote", tpath, "and", out / "features_ref_text.npz")


def _retrieval_cases():
    """(name, n_leaves, offsets, words, p_match, n_best)."""
    cases = []
    off, w = synth.sequence_words(11, n_images=48, n_leaves=2000, n_min=30, n_max=120, window=6, zipf=1.1)
    cases.append(("seq48", 2000, off, w, 0.1, 6))
    off, w = synth.sequence_words(12, n_images=70, n_leaves=5000, n_min=100, n_max=300, window=4, zipf=1.3)
    cases.append(("seq70_zipf", 5000, off, w, 0.05, 12))
    rng = np.random.default_rng(13)
    imgs = [rng.integers(0, 300, 40), np.zeros(0, np.int64), rng.integers(0, 300, 25)]
    imgs.append(imgs[0].copy())                       # identical to image 0
    imgs.append(imgs[0].copy())                       # and again: equal scores, ranked by index
    imgs.append(np.repeat(rng.integers(0, 300, 6), 7))  # repeated words
    imgs.append(np.arange(300, 330))                  # words no earlier image has
    imgs.append(rng.integers(0, 300, 1))
    imgs += [rng.integers(0, 300, int(n)) for n in rng.integers(5, 60, 12)]
    off = np.zeros(len(imgs) + 1, np.int32)
    off[1:] = np.cumsum([x.shape[0] for x in imgs])
    w = np.concatenate(imgs).astype(np.int32)
    cases.append(("edges", 400, off, w, 0.1, 5))
    cases.append(("edges_all", 400, off, w, 0.0, 40))  # n_best above the image count
    off1 = np.array([0, 3], np.int32)
    cases.append(("single", 10, off1, np.array([1, 2, 2], np.int32), 0.1, 3))
    return cases


def make_retrieval(out: Path) -> None:
    if not oracle.ref_retrieval_available():
        raise SystemExit("oracle/_ref/libv3dref_retrieval.so missing: run `make -C oracle ref` first")
    arrays = {}
    names = []
    for name, n_leaves, off, w, pm, nb in _retrieval_cases():
        docs, sc = oracle.ref_retrieval(n_leaves, off, w, pm, nb)
        assert np.isfinite(sc).all()
        names.append(name)
        arrays[f"{name}_n_leaves"] = np.array(n_leaves, np.int32)
        arrays[f"{name}_offsets"] = off.astype(np.int32)
        arrays[f"{name}_words"] = w.astype(np.int32)
        arrays[f"{name}_p_match"] = np.array(pm, np.float64)
        arrays[f"{name}_docs"] = docs
        arrays[f"{name}_scores"] = sc
        print(f"{name}: {off.shape[0] - 1} images, {w.shape[0]} words, n_best {nb}")
    arrays["names"] = np.array(names)
    np.savez_compressed(out / "retrieval_ref.npz", **arrays)
    print("wrote", out / "retrieval_ref.npz")


def make_ransac(out: Path) -> None:
    if not oracle.ref_ransac_available():
        raise SystemExit("oracle/_ref/libv3dref_ransac.so missing: run `make -C oracle ref` first")
    rng = np.random.default_rng(77)
    pts, sols, counts = [], [], []
    for t in range(300):
        if t % 2 == 0:
            v = rng.normal(size=3) * 0.3
            th = np.linalg.norm(v)
            k = v / th
            Kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
            R = np.eye(3) + np.sin(th) * Kx + (1 - np.cos(th)) * Kx @ Kx
            X = np.c_[rng.uniform(-1, 1, (5, 2)), rng.uniform(3, 6, 5)]
            p = X[:, :2] / X[:, 2:]
            Y = (R @ X.T).T + rng.normal(size=3)
            q = Y[:, :2] / Y[:, 2:]
        else:
            p = rng.uniform(-0.5, 0.5, (5, 2))
            q = rng.uniform(-0.5, 0.5, (5, 2))
        row = np.r_[p[:, 0], p[:, 1], q[:, 0], q[:, 1]]
        E = oracle.ref_five_point(row[:5], row[5:10], row[10:15], row[15:])
        E10 = np.zeros((10, 3, 3))
        E10[:len(E)] = E
        pts.append(row)
        sols.append(E10)
        counts.append(len(E))
    arrays = {"fp_pts": np.array(pts), "fp_E": np.array(sols), "fp_counts": np.array(counts, np.int32)}
    off, corrs, K, R, t, inl = synth.two_view_pairs(78, n_pairs=6, n_min=200, n_max=1200)
    models, nins, chosen, samples, flags = [], [], [], [], []
    for p in range(6):
        c = corrs[off[p]:off[p + 1]]
        s = oracle.ref_shuffle_samples(c.shape[0], 1000, 500 + p)
        res = oracle.ref_ransac(c, K[p, 0], K[p, 1], 2.0, 1000, s)
        models.append(res["model"])
        nins.append(res["n_inliers"])
        chosen.append(res["chosen"])
        samples.append(s)
        flags.append(res["flags"])
    arrays.update(rs_offsets=off, rs_corrs=corrs, rs_K=K, rs_models=np.array(models),
                  rs_n_inliers=np.array(nins, np.int32), rs_chosen=np.array(chosen, np.int32),
                  rs_flags=np.concatenate(flags), rs_seeds=np.arange(500, 506, dtype=np.int32))
    for p in range(6):
        arrays[f"rs_samples_{p}"] = samples[p]
    np.savez_compressed(out / "ransac_ref.npz", **arrays)
    print("wrote", out / "ransac_ref.npz", "solutions", int(np.sum(counts)), "chosen", chosen)


def main(argv):
    makers = {"voctree": make_voctree, "match": make_match, "features": make_features,
              "retrieval": make_retrieval, "ransac": make_ransac}
    if len(argv) < 2 or argv[1] not in makers:
        raise SystemExit(__doc__)
    out = Path(argv[2]) if len(argv) > 2 else HERE
    out.mkdir(parents=True, exist_ok=True)
    makers[argv[1]](out)


if __name__ == "__main__":
    main(sys.argv)
