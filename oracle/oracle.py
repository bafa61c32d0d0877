"""ctypes loader for the parity oracle (liboracle.so) and the reference builds in _ref/.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, never by the library.  See v3dm_oracle.c for what each function restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_VOCTREE = HERE / "_ref" / "libv3dref_voctree.so"
REF_CUDA = HERE / "_ref" / "libv3dref_cuda.so"
REF_FEATURES = HERE / "_ref" / "libv3dref_features.so"
REF_RETRIEVAL = HERE / "_ref" / "libv3dref_retrieval.so"
REF_RANSAC = HERE / "_ref" / "libv3dref_ransac.so"

_lib = None


class Gate(C.Structure):
    _fields_ = [("type", C.c_int), ("m", C.c_double * 9), ("thr", C.c_float)]


def ref_dir() -> Path:
    """The reference's V3D source tree: V3D_REF_DIR, else the reference checkout beside this
    repository."""
    return Path(os.environ.get("V3D_REF_DIR", str(HERE.parent.parent / "reference" / "V3D")))


def build() -> None:
    """Builds liboracle.so (and the _ref libraries when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if ref_dir().exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
        L.orc_match_u8.argtypes = [i32, i32, vp, vp, f32, f32, i32, vp, vp, vp, vp, vp, vp, i32]
        L.orc_match_u8.restype = i32
        L.orc_voctree_quantize_f32.argtypes = [i32, i32, vp, i32, vp, vp, i32, i32]
        L.orc_voctree_quantize_u8.argtypes = [i32, i32, vp, i32, vp, vp, i32, i32]
        L.orc_match_u8_calls.argtypes = [i32, i32, vp, vp, f32, f32, i32, vp, vp, vp, vp, vp, vp, i32]
        L.orc_match_u8_calls.restype = i32
        L.orc_scores_u8.argtypes = [i32, i32, vp, vp, vp]
        L.orc_ref_feature_count.argtypes = [i32, i32]
        L.orc_ref_feature_count.restype = i32
        L.orc_num_threads.restype = i32
        L.orc_retrieval_binomial.argtypes = [i32, i32, vp, vp, C.c_double, i32, vp, vp, i32]
        L.orc_retrieval_binomial.restype = i32
        _lib = L
    return _lib


def num_threads() -> int:
    return lib().orc_num_threads()


def _gates(gates):
    arr = (Gate * max(1, len(gates)))()
    for i, (typ, M, thr) in enumerate(gates):
        arr[i].type = 1 if typ in ("F", 1) else 2
        for k, v in enumerate(np.asarray(M, np.float64).reshape(9)):
            arr[i].m[k] = float(v)
        arr[i].thr = float(thr)
    return arr


def match(L: np.ndarray, R: np.ndarray, min_score: float = 0.9, min_ratio: float = 0.8, gates=(),
          lpos=None, rpos=None, threads: int = 0, with_sides: bool = False):
    """The reference's putative (no gates) or guided matching on uint8 descriptors.

    gates: sequence of ("F" | "H", 3x3 matrix, threshold); they compound as successive
    runGuidedMatching calls do.  Returns (n, 2) int32 pairs (left, right) ascending in left,
    plus the per-left and per-right results when with_sides."""
    L = np.ascontiguousarray(L, np.uint8)
    R = np.ascontiguousarray(R, np.uint8)
    nL, nR = L.shape[0], R.shape[0]
    g = _gates(list(gates))
    lp = np.ascontiguousarray(lpos, np.float32) if lpos is not None else np.zeros((1, 2), np.float32)
    rp = np.ascontiguousarray(rpos, np.float32) if rpos is not None else np.zeros((1, 2), np.float32)
    pairs = np.empty((max(1, min(nL, nR)), 2), np.int32)
    colmax = np.empty(max(1, nL), np.int32)
    rowmax = np.empty(max(1, nR), np.int32)
    n = lib().orc_match_u8(nL, nR, L.ctypes.data, R.ctypes.data, min_score, min_ratio, len(gates),
                           C.addressof(g), lp.ctypes.data, rp.ctypes.data, colmax.ctypes.data, rowmax.ctypes.data,
                           pairs.ctypes.data, threads)
    if n < 0:
        raise ValueError("oracle rejected the arguments")
    out = pairs[:n].copy()
    if with_sides:
        return out, colmax[:nL].copy(), rowmax[:nR].copy()
    return out


def match_calls(L: np.ndarray, R: np.ndarray, min_score: float, min_ratio: float, calls, lpos=None, rpos=None,
                threads: int = 0):
    """A putative call and guided calls on the same features from one score computation, as
    the reference's guided calls mask the putative call's stored matrix.  calls: a list of
    gate lists, one per call, each extending the previous one (gates compound); the first is
    normally [] (putative).  Returns one (n, 2) pair array per call."""
    L = np.ascontiguousarray(L, np.uint8)
    R = np.ascontiguousarray(R, np.uint8)
    nL, nR = L.shape[0], R.shape[0]
    calls = [list(c) for c in calls]
    for a, b in zip(calls, calls[1:]):
        if b[:len(a)] != a:
            raise ValueError("each call's gates must extend the previous call's")
    g = _gates(calls[-1])
    upto = np.array([len(c) for c in calls], np.int32)
    lp = np.ascontiguousarray(lpos, np.float32) if lpos is not None else np.zeros((1, 2), np.float32)
    rp = np.ascontiguousarray(rpos, np.float32) if rpos is not None else np.zeros((1, 2), np.float32)
    cap = max(1, min(nL, nR))
    pairs = np.empty((len(calls), cap, 2), np.int32)
    n_out = np.zeros(len(calls), np.int32)
    rc = lib().orc_match_u8_calls(nL, nR, L.ctypes.data, R.ctypes.data, min_score, min_ratio, len(calls),
                                  upto.ctypes.data, C.addressof(g), lp.ctypes.data, rp.ctypes.data,
                                  pairs.ctypes.data, n_out.ctypes.data, threads)
    if rc != 0:
        raise ValueError("oracle rejected the arguments")
    return [pairs[c, :n_out[c]].copy() for c in range(len(calls))]


def scores(L: np.ndarray, R: np.ndarray) -> np.ndarray:
    """Integer score matrix S[r, l] (small cases)."""
    L = np.ascontiguousarray(L, np.uint8)
    R = np.ascontiguousarray(R, np.uint8)
    S = np.empty((R.shape[0], L.shape[0]), np.int32)
    lib().orc_scores_u8(L.shape[0], R.shape[0], L.ctypes.data, R.ctypes.data, S.ctypes.data)
    return S


def voctree(bf: int, depth: int, nodes: np.ndarray, keys: np.ndarray, global_ids: bool = True,
            threads: int = 0) -> np.ndarray:
    keys_c = np.ascontiguousarray(keys)
    nodes_c = np.ascontiguousarray(nodes)
    out = np.empty(keys_c.shape[0], np.int32)
    if keys_c.dtype == np.uint8:
        rc = lib().orc_voctree_quantize_u8(bf, depth, nodes_c.ctypes.data, keys_c.shape[0], keys_c.ctypes.data,
                                           out.ctypes.data, int(global_ids), threads)
    else:
        nodes_c = np.ascontiguousarray(nodes_c, np.float32)
        keys_c = np.ascontiguousarray(keys_c, np.float32)
        rc = lib().orc_voctree_quantize_f32(bf, depth, nodes_c.ctypes.data, keys_c.shape[0], keys_c.ctypes.data,
                                            out.ctypes.data, int(global_ids), threads)
    if rc != 0:
        raise ValueError("oracle rejected the arguments")
    return out


def retrieval(n_leaves: int, offsets: np.ndarray, words: np.ndarray, p_match: float, n_best: int,
              threads: int = 0):
    """The voctree app's image loop over LeafDocuments::computeBinomialScores (restated):
    (best_docs, best_scores), nImages x n_best, -1 / 0 past the i-th entry of row i."""
    off = np.ascontiguousarray(offsets, np.int32)
    w = np.ascontiguousarray(words, np.int32)
    n = off.shape[0] - 1
    docs = np.empty((n, n_best), np.int32)
    sc = np.empty((n, n_best), np.float32)
    if lib().orc_retrieval_binomial(n_leaves, n, off.ctypes.data, w.ctypes.data, float(p_match), n_best,
                                    docs.ctypes.data, sc.ctypes.data, threads) != 0:
        raise ValueError("oracle rejected the arguments")
    return docs, sc


def ref_feature_count(n: int, n_max_rounded: int) -> int:
    return lib().orc_ref_feature_count(n, n_max_rounded)


# ---- the reference's own code ---------------------------------------------------------------

def ref_voctree_available() -> bool:
    return REF_VOCTREE.exists()


def ref_voctree(bf: int, depth: int, nodes_f32: np.ndarray, keys_f32: np.ndarray) -> np.ndarray:
    """V3D::VocabularyTree<depth, bf, 128>::getVisualWord (leaf-local ids), compiled from the
    reference headers."""
    L = C.CDLL(str(REF_VOCTREE))
    L.v3dref_voctree_quantize.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    n = np.ascontiguousarray(nodes_f32, np.float32)
    k = np.ascontiguousarray(keys_f32, np.float32)
    out = np.empty(k.shape[0], np.int32)
    rc = L.v3dref_voctree_quantize(bf, depth, n.ctypes.data, k.shape[0], k.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"shape BF={bf} D={depth} not instantiated in ref_voctree_wrap.cpp")
    return out


def ref_cuda_available() -> bool:
    return REF_CUDA.exists()


_REF_CHILD = r"""
import ctypes as C, sys, numpy as np
d = np.load(sys.argv[1])
L = C.CDLL(sys.argv[2])
L.v3dref_match.argtypes = [C.c_int]*4 + [C.c_void_p]*2 + [C.c_float]*2 + [C.c_int] + [C.c_void_p]*6 + [C.c_void_p]
Lf = np.ascontiguousarray(d['L'], np.float32); Rf = np.ascontiguousarray(d['R'], np.float32)
gt = np.ascontiguousarray(d['gtypes'], np.int32); gm = np.ascontiguousarray(d['gmats'], np.float64)
gth = np.ascontiguousarray(d['gthr'], np.float32)
lp = np.ascontiguousarray(d['lpos'], np.float32); rp = np.ascontiguousarray(d['rpos'], np.float32)
nL, nR = Lf.shape[0], Rf.shape[0]
pairs = np.empty((max(1, min(nL, nR)), 2), np.int32); nput = C.c_int(0)
n = L.v3dref_match(int(d['nmaxl']), int(d['nmaxr']), nL, nR, Lf.ctypes.data, Rf.ctypes.data,
                   float(d['ms']), float(d['mr']), int(gt.size), gt.ctypes.data, gm.ctypes.data, gth.ctypes.data,
                   lp.ctypes.data, rp.ctypes.data, pairs.ctypes.data, C.byref(nput))
np.save(sys.argv[3], pairs[:max(n, 0)])
sys.exit(0 if n >= 0 else 3)
"""


def ref_cuda_match(L_u8: np.ndarray, R_u8: np.ndarray, min_score: float, min_ratio: float, gates=(),
                   lpos=None, rpos=None, workdir: str | None = None) -> np.ndarray:
    """The reference's own SIFT_Matching (v3d_cudamatching.cu) on a GPU, fed u/512 floats.
    Runs in a child process because the reference exits on any CUDA error.  Sizes must be
    multiples of 32 (the reference's own requirement)."""
    return ref_cuda_match_f32(L_u8.astype(np.float32) / 512.0, R_u8.astype(np.float32) / 512.0, min_score,
                              min_ratio, gates, lpos, rpos, workdir)


def ref_cuda_match_f32(L_f32: np.ndarray, R_f32: np.ndarray, min_score: float, min_ratio: float, gates=(),
                       lpos=None, rpos=None, workdir: str | None = None) -> np.ndarray:
    """The reference's own SIFT_Matching on arbitrary float descriptors (its FP32 cublasSgemm
    scores, built with --use_fast_math as the reference builds it)."""
    import tempfile
    wd = Path(workdir or tempfile.mkdtemp(prefix="v3dref_"))
    wd.mkdir(parents=True, exist_ok=True)
    gates = list(gates)
    nL, nR = L_f32.shape[0], R_f32.shape[0]
    np.savez(wd / "in.npz", L=np.asarray(L_f32, np.float32), R=np.asarray(R_f32, np.float32),
             gtypes=np.array([1 if t in ("F", 1) else 2 for t, _, _ in gates], np.int32),
             gmats=np.array([np.asarray(M, np.float64).reshape(9) for _, M, _ in gates], np.float64).reshape(-1),
             gthr=np.array([thr for _, _, thr in gates], np.float32),
             lpos=np.zeros((nL, 2), np.float32) if lpos is None else lpos,
             rpos=np.zeros((nR, 2), np.float32) if rpos is None else rpos,
             nmaxl=nL, nmaxr=nR, ms=min_score, mr=min_ratio)
    res = subprocess.run([sys.executable, "-c", _REF_CHILD, str(wd / "in.npz"), str(REF_CUDA), str(wd / "out.npy")],
                         capture_output=True, text=True, timeout=600)
    if res.returncode != 0:
        raise RuntimeError(f"reference matcher failed ({res.returncode}): {res.stderr[-2000:]}")
    return np.load(wd / "out.npy")


_REF_TIME_CHILD = r"""
import ctypes as C, json, sys, numpy as np
d = np.load(sys.argv[1])
L = C.CDLL(sys.argv[2])
L.v3dref_time_pairs.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 3 + [C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
off = np.ascontiguousarray(d['off'], np.int32); desc = np.ascontiguousarray(d['desc'], np.float32)
pos = np.ascontiguousarray(d['pos'], np.float32); pairs = np.ascontiguousarray(d['pairs'], np.int32)
F = np.ascontiguousarray(d['F'], np.float64); reps = int(d['reps'])
sec = np.zeros(reps, np.float64); nm = C.c_longlong(0)
rc = L.v3dref_time_pairs(int(d['nmax']), off.size - 1, off.ctypes.data, desc.ctypes.data, pos.ctypes.data,
                         pairs.shape[0], pairs.ctypes.data, int(d['guided']), F.ctypes.data, float(d['thr']),
                         float(d['ms']), float(d['mr']), reps, sec.ctypes.data, C.byref(nm))
print(json.dumps({"rc": rc, "seconds": sec.tolist(), "matches": nm.value}))
sys.exit(0 if rc == 0 else 3)
"""


def ref_cuda_time_pairs(desc_u8: np.ndarray, offsets: np.ndarray, pairs: np.ndarray, min_score: float,
                        min_ratio: float, reps: int, positions=None, F=None, thr: float = 2.0,
                        n_max: int | None = None, timeout: float = 900.0) -> dict:
    """Wall time of the reference's own SIFT_Matching (v3d_cudamatching.cu, built unmodified
    for the B200) in the apps' per-pair loop over `pairs` of the images in desc_u8 (u/512
    floats), with F-guided matching after each putative call when F (9 doubles per pair) is
    given.  Runs in a child process because the reference exits on any CUDA error.
    Returns {"seconds": [per repetition], "matches": pairs found in the last repetition}."""
    import json
    import tempfile
    wd = Path(tempfile.mkdtemp(prefix="v3dref_time_"))
    off = np.ascontiguousarray(offsets, np.int32)
    counts = np.diff(off)
    guided = F is not None
    np.savez(wd / "in.npz", off=off, desc=np.asarray(desc_u8, np.float32) / 512.0,
             pos=np.zeros((max(1, off[-1]), 2), np.float32) if positions is None else positions,
             pairs=np.ascontiguousarray(pairs, np.int32).reshape(-1, 2),
             F=np.zeros(9, np.float64) if F is None else np.asarray(F, np.float64).reshape(-1),
             guided=int(guided), thr=thr, ms=min_score, mr=min_ratio, reps=reps,
             nmax=int(n_max if n_max is not None else (int(counts.max()) & ~31)))
    res = subprocess.run([sys.executable, "-c", _REF_TIME_CHILD, str(wd / "in.npz"), str(REF_CUDA)],
                         capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"reference matcher failed ({res.returncode}): {res.stderr[-2000:]}")
    return json.loads(res.stdout.strip().splitlines()[-1])


# ---- the reference's feature-file serializer -------------------------------------------------

FEATURE_FIELDS = ("ids", "positions", "directions", "scales", "magnitudes", "descriptors")


def ref_features_available() -> bool:
    return REF_FEATURES.exists()


def _ref_features_lib():
    L = C.CDLL(str(REF_FEATURES))
    L.ref_features_write.argtypes = [C.c_char_p, C.c_int] + [C.c_void_p] * 6
    L.ref_features_write_as.argtypes = [C.c_char_p, C.c_int, C.c_int] + [C.c_void_p] * 6
    L.ref_features_read.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int)] + [C.c_void_p] * 6
    return L


def ref_features_write(path: str, f: dict, binary: bool = True) -> None:
    """serializeDataToFile(path, SerializableVector<SIFT_Feature>, binary) of the reference
    (binary: "V3DBIN", else the text archive "V3DTXT")."""
    L = _ref_features_lib()
    n = f["ids"].shape[0]
    a = [np.ascontiguousarray(f[k], np.int32 if k == "ids" else np.float32) for k in FEATURE_FIELDS]
    if L.ref_features_write_as(str(path).encode(), int(binary), n, *[x.ctypes.data for x in a]) != 0:
        raise OSError(f"reference writer failed on {path}")


def ref_features_count(path: str) -> int:
    """One full serializeDataFromFile of the reference; returns the feature count (the arrays are
    not copied out)."""
    L = _ref_features_lib()
    n = C.c_int(0)
    if L.ref_features_read(str(path).encode(), 0, C.byref(n), *([None] * 6)) != 0:
        raise OSError(f"reference reader failed on {path}")
    return n.value


def ref_features_read(path: str) -> dict:
    """serializeDataFromFile(path, SerializableVector<SIFT_Feature>&) of the reference.  Only for
    well-formed files: on a malformed text archive the reference's reader throws from a
    destructor, which ends the process."""
    L = _ref_features_lib()
    n = C.c_int(0)
    if L.ref_features_read(str(path).encode(), 0, C.byref(n), *([None] * 6)) != 0:
        raise OSError(f"reference reader failed on {path}")
    m = n.value
    out = {"ids": np.empty(m, np.int32), "positions": np.empty((m, 2), np.float32),
           "directions": np.empty((m, 2), np.float32), "scales": np.empty(m, np.float32),
           "magnitudes": np.empty(m, np.float32), "descriptors": np.empty((m, 128), np.float32)}
    if L.ref_features_read(str(path).encode(), m, C.byref(n), *[out[k].ctypes.data for k in FEATURE_FIELDS]) != 0:
        raise OSError(f"reference reader failed on {path}")
    return out


# ---- the reference's inverted files ---------------------------------------------------------

def ref_retrieval_available() -> bool:
    return REF_RETRIEVAL.exists()


def ref_retrieval(n_leaves: int, offsets: np.ndarray, words: np.ndarray, p_match: float, n_best: int):
    """The image loop of match_using_voctree.cpp:176-222 on the reference's LeafDocuments
    (computeBinomialScores, then insertDocument), one thread.  Same outputs as retrieval()."""
    L = C.CDLL(str(REF_RETRIEVAL))
    L.ref_retrieval.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                                C.c_void_p]
    off = np.ascontiguousarray(offsets, np.int32)
    w = np.ascontiguousarray(words, np.int32)
    n = off.shape[0] - 1
    docs = np.empty((n, n_best), np.int32)
    sc = np.empty((n, n_best), np.float32)
    if L.ref_retrieval(n_leaves, n, off.ctypes.data, w.ctypes.data, float(p_match), n_best, docs.ctypes.data,
                       sc.ctypes.data) != 0:
        raise ValueError("reference retrieval failed")
    return docs, sc


def ref_retrieval_sampled(n_leaves: int, offsets: np.ndarray, words: np.ndarray, p_match: float, n_best: int,
                          stride: int, phase: int = 0):
    """The reference's loop with every image inserted and the images i % stride == phase
    queried: (seconds of those queries, seconds of all insertions, number of queries, sum of
    their best documents' ids)."""
    L = C.CDLL(str(REF_RETRIEVAL))
    L.ref_retrieval_sampled.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int,
                                        C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    off = np.ascontiguousarray(offsets, np.int32)
    w = np.ascontiguousarray(words, np.int32)
    tq, ti, nq, cs = C.c_double(), C.c_double(), C.c_int(), C.c_longlong()
    L.ref_retrieval_sampled(n_leaves, off.shape[0] - 1, off.ctypes.data, w.ctypes.data, float(p_match), n_best,
                            stride, phase, C.byref(tq), C.byref(ti), C.byref(nq), C.byref(cs))
    return tq.value, ti.value, nq.value, cs.value


# ---- the reference's relative orientation ---------------------------------------------------

def ref_ransac_available() -> bool:
    return REF_RANSAC.exists()


def _ref_ransac_lib():
    L = C.CDLL(str(REF_RANSAC))
    vp = C.c_void_p
    L.ref_five_point.argtypes = [vp] * 5 + [C.POINTER(C.c_int)]
    L.ref_pose.argtypes = [vp] * 7
    L.ref_shuffle_samples.argtypes = [C.c_int, C.c_int, C.c_uint, C.c_int, vp, C.POINTER(C.c_int)]
    L.ref_ransac.argtypes = [C.c_int, vp, vp, vp, C.c_double, C.c_int, C.c_int, vp, vp, C.POINTER(C.c_int), vp,
                             C.POINTER(C.c_int)]
    L.ref_ransac_mode.argtypes = [C.c_int, vp, vp, vp, C.c_double, C.c_int, C.c_int, vp, C.c_int, vp,
                                  C.POINTER(C.c_int), vp, C.POINTER(C.c_int)]
    L.ref_ransac_swap.argtypes = [C.c_int, vp, vp, vp, C.c_double, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp,
                                  C.POINTER(C.c_int), vp, C.POINTER(C.c_int)]
    return L


# ref_ransac(swap=...): the library's restatements in place of the reference's components.
SWAP_SOLVER, SWAP_POSE, SWAP_REFINE = 1, 2, 4


def ref_five_point(x1, y1, x2, y2):
    """computeEssentialsFromFiveCorrs: (k, 3, 3) essential matrices."""
    L = _ref_ransac_lib()
    a = [np.ascontiguousarray(v, np.float64) for v in (x1, y1, x2, y2)]
    E = np.zeros(90)
    n = C.c_int(0)
    L.ref_five_point(*[v.ctypes.data for v in a], E.ctypes.data, C.byref(n))
    return E[:9 * n.value].reshape(-1, 3, 3)


def ref_shuffle_samples(n: int, n_samples: int, seed: int) -> np.ndarray:
    L = _ref_ransac_lib()
    out = np.empty((n_samples + 1, 5), np.int32)
    nd = C.c_int(0)
    L.ref_shuffle_samples(n, n_samples, seed, n_samples + 1, out.ctypes.data, C.byref(nd))
    return out[:nd.value].copy()


def ref_ransac(corrs: np.ndarray, K1: np.ndarray, K2: np.ndarray, inlier_threshold: float, n_samples: int,
               samples: np.ndarray, refine: bool = False, swap: int = 0):
    """The loop of computeRobustOrientationMLE on one pair with the given samples, without
    (default) or with mode.iterativeRefinement: dict(model (31), n_inliers, flags,
    chosen = sample * 10 + solution index or -1).  swap (SWAP_* bits) replaces the reference's
    five-point solver, pose recovery or refinement by the library's restatement; all three give
    the GPU's algorithm on the CPU."""
    L = _ref_ransac_lib()
    c = np.ascontiguousarray(corrs, np.float32).reshape(-1, 4)
    k1 = np.ascontiguousarray(K1, np.float64)
    k2 = np.ascontiguousarray(K2, np.float64)
    s = np.ascontiguousarray(samples, np.int32).reshape(-1, 5)
    model = np.empty(31)
    nin, ch = C.c_int(0), C.c_int(0)
    flags = np.empty(c.shape[0], np.uint8)
    L.ref_ransac_swap(c.shape[0], c.ctypes.data, k1.ctypes.data, k2.ctypes.data, float(inlier_threshold), n_samples,
                      s.shape[0], s.ctypes.data, int(refine), int(swap), model.ctypes.data, C.byref(nin),
                      flags.ctypes.data, C.byref(ch))
    return {"model": model, "n_inliers": nin.value, "flags": flags, "chosen": ch.value}
