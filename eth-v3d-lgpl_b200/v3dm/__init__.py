"""Python mirror of the reference's matching interface over the C ABI of libv3dm.so.

``SIFTMatching`` follows ``V3D_CUDA::SIFT_Matching`` (V3D/CUDA/v3d_cudamatching.h:15-67) and
``VocabularyTreeTraversal`` follows ``V3D_CUDA::VocabularyTreeTraversal<BF, Depth>``
(v3d_cudamatching.h:69-105): same member names in snake_case, same argument meaning and
defaults (minScore 0.9, minRatio 0.8).  Where the reference prints and exits
(v3d_cudamatching.cu:12-27) this wrapper raises ``V3DMError``.  The library has no CPU
path: without the built libv3dm.so or without an sm_100 GPU every compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_DIR / "libv3dm.so"
HEADER_PATH = PKG_DIR.parent / "include" / "v3dm.h"

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_NOT_ALLOCATED = 3
ERR_SIZE = 4
ERR_CAPACITY = 5
ERR_NOT_U8 = 6
ERR_UNSUPPORTED = 7
ERR_TIMEOUT = 8
ERR_NO_DEVICE = 9
ERR_CANDIDATES = 10

KERNEL_TCGEN05 = 0
KERNEL_SIMT = 1
LEAF_GLOBAL = 0
LEAF_LOCAL = 1
MAX_FEATURES = 131072
MAX_GATES = 8

_lib = None


class V3DMError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().v3dm_status_string(status).decode() if _lib is not None else str(status)
        if status == ERR_CUDA and _lib is not None:
            msg += " [" + lib().v3dm_last_error().decode() + "]"
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


def lib() -> C.CDLL:
    """The loaded libv3dm.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"libv3dm.so not built ({LIB_PATH}); run __graft_entry__.build()")
        L = C.CDLL(str(LIB_PATH))
        vp, i32, f32, f64p = C.c_void_p, C.c_int, C.c_float, C.POINTER(C.c_double)
        L.v3dm_status_string.restype = C.c_char_p
        L.v3dm_status_string.argtypes = [i32]
        L.v3dm_last_error.restype = C.c_char_p
        L.v3dm_last_error.argtypes = []
        L.v3dm_matcher_create.argtypes = [C.POINTER(vp), i32, C.c_uint]
        L.v3dm_matcher_destroy.argtypes = [vp]
        L.v3dm_allocate.argtypes = [vp, i32, i32, i32]
        L.v3dm_deallocate.argtypes = [vp]
        for n in ("v3dm_set_left_f32", "v3dm_set_right_f32", "v3dm_set_left_u8", "v3dm_set_right_u8",
                  "v3dm_set_left_f32_bf16x3", "v3dm_set_right_f32_bf16x3", "v3dm_set_left_u8_device",
                  "v3dm_set_right_u8_device", "v3dm_set_left_f32_device", "v3dm_set_right_f32_device"):
            getattr(L, n).argtypes = [vp, i32, vp]
        L.v3dm_features_read.argtypes = [C.c_char_p, i32, C.POINTER(i32)] + [vp] * 6
        L.v3dm_quantize_u8_device.argtypes = [vp, C.c_longlong, vp, vp]
        L.v3dm_loader_create.argtypes = [i32, C.POINTER(vp)]
        L.v3dm_loader_destroy.argtypes = [vp]
        L.v3dm_loader_load.argtypes = [vp, i32, C.POINTER(C.c_char_p), i32, i32, vp]
        L.v3dm_loader_positions.argtypes = [vp, vp]
        L.v3dm_loader_descriptors_device.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_longlong)]
        L.v3dm_loader_descriptors_f32_device.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_longlong)]
        L.v3dm_loader_exact_u8.argtypes = [vp, C.POINTER(i32)]
        L.v3dm_scores_f32.argtypes = [vp, vp]
        L.v3dm_float_threshold.argtypes = [f32, f32, C.POINTER(C.c_float)]
        L.v3dm_putative.argtypes = [vp, f32, f32, vp, i32, C.POINTER(i32)]
        for n in ("v3dm_guided_F", "v3dm_guided_H"):
            getattr(L, n).argtypes = [vp, f64p, f32, vp, vp, f32, f32, vp, i32, C.POINTER(i32)]
        L.v3dm_putative_device.argtypes = [vp, f32, f32, vp, vp]
        L.v3dm_guided_F_device.argtypes = [vp, f64p, f32, vp, vp, f32, f32, vp, vp]
        L.v3dm_matcher_stream.argtypes = [vp, C.POINTER(vp)]
        L.v3dm_matcher_wait.argtypes = [vp]
        L.v3dm_matcher_last_launches.argtypes = [vp, C.POINTER(i32)]
        L.v3dm_matcher_profile.argtypes = [vp, i32]
        L.v3dm_matcher_num_configs.argtypes = [vp, C.POINTER(i32)]
        L.v3dm_matcher_get_config.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
        L.v3dm_matcher_set_config.argtypes = [vp, i32]
        L.v3dm_matcher_test_wait_fault.argtypes = [vp, C.c_longlong, i32]
        L.v3dm_matcher_autotune.argtypes = [vp, f32, f32, i32, C.POINTER(i32), C.POINTER(C.c_double)]
        L.v3dm_matcher_profile_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(i32)]
        L.v3dm_matcher_profile_read_pass.argtypes = [vp, i32, C.POINTER(C.c_double), C.POINTER(i32)]
        L.v3dm_candidate_threshold.argtypes = [f32, f32, i32, C.POINTER(C.c_int32)]
        L.v3dm_voctree_create.argtypes = [C.POINTER(vp), i32, i32, i32]
        L.v3dm_voctree_destroy.argtypes = [vp]
        L.v3dm_voctree_counts.argtypes = [i32, i32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.v3dm_voctree_allocate.argtypes = [vp, i32]
        L.v3dm_voctree_set_nodes_f32.argtypes = [vp, vp]
        L.v3dm_voctree_set_nodes_u8.argtypes = [vp, vp]
        L.v3dm_voctree_quantize_f32.argtypes = [vp, i32, vp, vp, i32]
        L.v3dm_voctree_quantize_u8.argtypes = [vp, i32, vp, vp, i32]
        L.v3dm_voctree_quantize_u8_device.argtypes = [vp, i32, vp, vp, i32]
        L.v3dm_voctree_quantize_f32_device.argtypes = [vp, i32, vp, vp, i32]
        L.v3dm_voctree_replays.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.v3dm_voctree_stream.argtypes = [vp, C.POINTER(vp)]
        L.v3dm_voctree_last_launches.argtypes = [vp, C.POINTER(i32)]
        i64, i64p = C.c_longlong, C.POINTER(C.c_longlong)
        L.v3dm_batch_create.argtypes = [C.POINTER(vp), i32]
        L.v3dm_batch_destroy.argtypes = [vp]
        L.v3dm_batch_set_images_u8.argtypes = [vp, i32, vp, vp]
        L.v3dm_batch_set_images_u8_device.argtypes = [vp, i32, vp, vp]
        L.v3dm_batch_set_images_f32.argtypes = [vp, i32, vp, vp]
        L.v3dm_batch_set_images_f32_device.argtypes = [vp, i32, vp, vp]
        L.v3dm_batch_float_mode.argtypes = [vp, C.POINTER(i32)]
        L.v3dm_batch_set_pairs.argtypes = [vp, i32, vp]
        L.v3dm_batch_match.argtypes = [vp, f32, f32, vp, i64, i64p]
        L.v3dm_batch_match_device.argtypes = [vp, f32, f32, vp]
        L.v3dm_batch_set_positions.argtypes = [vp, vp]
        L.v3dm_batch_set_positions_device.argtypes = [vp, vp]
        L.v3dm_batch_match_guided.argtypes = [vp, i32, vp, vp, f32, f32, vp, i64, i64p]
        L.v3dm_batch_wait.argtypes = [vp]
        L.v3dm_batch_result_device.argtypes = [vp, C.POINTER(vp)]
        L.v3dm_batch_stream.argtypes = [vp, C.POINTER(vp)]
        L.v3dm_batch_use_graph.argtypes = [vp, i32]
        L.v3dm_batch_set_config.argtypes = [vp, i32, i32]
        L.v3dm_batch_get_config.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
        L.v3dm_batch_autotune.argtypes = [vp, f32, f32, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(C.c_float)]
        L.v3dm_batch_profile.argtypes = [vp, i32]
        L.v3dm_batch_profile_read.argtypes = [vp, i32, C.POINTER(C.c_double), C.POINTER(i32)]
        L.v3dm_batch_last_launches.argtypes = [vp, C.POINTER(i32)]
        L.v3dm_batch_work.argtypes = [vp, i64p, i64p]
        fp = C.POINTER(C.c_float)
        L.v3dm_projection_create.argtypes = [C.POINTER(vp), i32, C.c_ulonglong]
        L.v3dm_projection_destroy.argtypes = [vp]
        L.v3dm_projection_get_params.argtypes = [vp, vp]
        L.v3dm_projection_set_params.argtypes = [vp, vp]
        L.v3dm_projection_loss_grad.argtypes = [vp, vp, vp, i32, f32, fp, vp]
        L.v3dm_projection_train_step.argtypes = [vp, vp, vp, i32, f32, f32, fp]
        L.v3dm_projection_embed.argtypes = [vp, vp, i32, vp]
        L.v3dm_projection_set_cells.argtypes = [vp, i32, vp]
        L.v3dm_projection_assign.argtypes = [vp, vp, i32, i32, vp]
        L.v3dm_batch_match_proposal.argtypes = [vp, vp, i32, i32, f32, f32, vp, i64, i64p]
        L.v3dm_batch_match_proposal_device.argtypes = [vp, vp, i32, i32, f32, f32, vp]
        L.v3dm_batch_proposal_scored.argtypes = [vp, i64p, i64p]
        L.v3dm_retrieval_create.argtypes = [C.POINTER(vp), i32]
        L.v3dm_retrieval_destroy.argtypes = [vp]
        L.v3dm_retrieval_binomial.argtypes = [vp, i32, i32, vp, vp, C.c_double, i32, vp, vp]
        L.v3dm_retrieval_binomial_device.argtypes = [vp, i32, i32, vp, vp, C.c_double, i32, vp, vp]
        L.v3dm_retrieval_wait.argtypes = [vp]
        L.v3dm_retrieval_stream.argtypes = [vp, C.POINTER(vp)]
        L.v3dm_retrieval_pairs.argtypes = [i32, i32, vp, i64, vp, i64p]
        L.v3dm_ransac_create.argtypes = [C.POINTER(vp), i32]
        L.v3dm_ransac_destroy.argtypes = [vp]
        L.v3dm_ransac_essential.argtypes = [vp, i32, vp, vp, vp, C.c_double, i32, i32, vp, C.c_uint64, vp, vp, vp]
        L.v3dm_ransac_essential_device.argtypes = [vp, i32, vp, vp, vp, C.c_double, i32, i32, vp, C.c_uint64, vp,
                                                   vp, vp]
        L.v3dm_ransac_wait.argtypes = [vp]
        L.v3dm_ransac_set_refinement.argtypes = [vp, i32]
        L.v3dm_ransac_profile.argtypes = [vp, i32]
        L.v3dm_ransac_candidates.argtypes = [vp, i64p, i64p]
        L.v3dm_ransac_profile_read.argtypes = [vp, i32, C.POINTER(C.c_double), C.POINTER(i32)]
        L.v3dm_ransac_shuffle_samples.argtypes = [i32, i32, C.c_uint, i32, vp, C.POINTER(i32)]
        L.v3dm_essential_five_point.argtypes = [vp, i32, vp, vp, vp]
        L.v3dm_ransac_stream.argtypes = [vp, C.POINTER(vp)]
        L.v3dm_ransac_last_launches.argtypes = [vp, C.POINTER(i32)]
        L.v3dm_retrieval_profile.argtypes = [vp, i32]
        L.v3dm_retrieval_profile_read.argtypes = [vp, i32, C.POINTER(C.c_double), C.POINTER(i32)]
        _lib = L
    return _lib


def _check(status: int, what: str) -> None:
    if status != OK:
        raise V3DMError(status, what)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def candidate_threshold(min_score: float, min_ratio: float, gated: bool) -> int:
    """Candidate threshold T of the fused selection (host computation, no GPU needed)."""
    t = C.c_int32(0)
    _check(lib().v3dm_candidate_threshold(min_score, min_ratio, int(gated), C.byref(t)), "candidate_threshold")
    return t.value


def float_threshold(min_score: float, min_ratio: float) -> float:
    """Float candidate threshold of the BF16 hi/lo path (host computation, no GPU needed)."""
    t = C.c_float(0)
    _check(lib().v3dm_float_threshold(min_score, min_ratio, C.byref(t)), "float_threshold")
    return t.value


def _desc(desc: np.ndarray):
    d = np.ascontiguousarray(desc)
    if d.ndim != 2 or d.shape[1] != 128:
        raise ValueError("descriptors must be an (n, 128) array")
    if d.dtype == np.uint8:
        return d, "u8"
    return np.ascontiguousarray(d, dtype=np.float32), "f32"


def _pos(pos: np.ndarray, n: int) -> np.ndarray:
    p = np.ascontiguousarray(pos, dtype=np.float32)
    if p.shape != (n, 2):
        raise ValueError(f"positions must be ({n}, 2)")
    return p


class SIFTMatching:
    """V3D_CUDA::SIFT_Matching over libv3dm.so (one CUDA stream per instance)."""

    def __init__(self, device: int = 0, kernel: int = KERNEL_TCGEN05):
        h = C.c_void_p()
        _check(lib().v3dm_matcher_create(C.byref(h), device, kernel), "SIFT_Matching()")
        self._h = h
        self.kernel = kernel
        self.n_left = 0
        self.n_right = 0

    def close(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.v3dm_matcher_destroy(self._h)
        self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def allocate(self, n_max_left: int, n_max_right: int | None = None, use_guided_matching: bool = False):
        """SIFT_Matching::allocate (v3d_cudamatching.h:33-37); sizes used as given."""
        if n_max_right is None:
            n_max_right = n_max_left
        _check(lib().v3dm_allocate(self._h, int(n_max_left), int(n_max_right), int(use_guided_matching)), "allocate")

    def deallocate(self):
        _check(lib().v3dm_deallocate(self._h), "deallocate")

    def set_left_features(self, desc: np.ndarray):
        d, kind = _desc(desc)
        fn = lib().v3dm_set_left_u8 if kind == "u8" else lib().v3dm_set_left_f32
        _check(fn(self._h, d.shape[0], _ptr(d)), "setLeftFeatures")
        self.n_left = d.shape[0]

    def set_right_features(self, desc: np.ndarray):
        d, kind = _desc(desc)
        fn = lib().v3dm_set_right_u8 if kind == "u8" else lib().v3dm_set_right_f32
        _check(fn(self._h, d.shape[0], _ptr(d)), "setRightFeatures")
        self.n_right = d.shape[0]

    def set_left_features_device(self, d_desc: int, n: int):
        """u8 descriptors already in device memory (v3dm_set_left_u8_device)."""
        _check(lib().v3dm_set_left_u8_device(self._h, n, C.c_void_p(d_desc)), "setLeftFeatures")
        self.n_left = n

    def set_right_features_device(self, d_desc: int, n: int):
        _check(lib().v3dm_set_right_u8_device(self._h, n, C.c_void_p(d_desc)), "setRightFeatures")
        self.n_right = n

    def set_left_features_f32_device(self, d_desc: int, n: int):
        """Float descriptors already in device memory (v3dm_set_left_f32_device): u/512 values
        take the exact integer path, others the BF16 hi/lo path."""
        _check(lib().v3dm_set_left_f32_device(self._h, n, C.c_void_p(d_desc)), "setLeftFeatures")
        self.n_left = n

    def set_right_features_f32_device(self, d_desc: int, n: int):
        _check(lib().v3dm_set_right_f32_device(self._h, n, C.c_void_p(d_desc)), "setRightFeatures")
        self.n_right = n

    def set_left_features_bf16x3(self, desc: np.ndarray):
        """Float descriptors scored with the BF16 hi/lo split whatever their values."""
        d = np.ascontiguousarray(desc, dtype=np.float32)
        _check(lib().v3dm_set_left_f32_bf16x3(self._h, d.shape[0], _ptr(d)), "setLeftFeatures(bf16x3)")
        self.n_left = d.shape[0]

    def set_right_features_bf16x3(self, desc: np.ndarray):
        d = np.ascontiguousarray(desc, dtype=np.float32)
        _check(lib().v3dm_set_right_f32_bf16x3(self._h, d.shape[0], _ptr(d)), "setRightFeatures(bf16x3)")
        self.n_right = d.shape[0]

    def scores_f32(self) -> np.ndarray:
        """BF16 hi/lo scores of the current descriptors, (n_left, n_right) float32."""
        out = np.empty((self.n_left, self.n_right), np.float32)
        _check(lib().v3dm_scores_f32(self._h, _ptr(out)), "scores_f32")
        return out

    def _result(self, fn, *args) -> np.ndarray:
        cap = max(1, min(self.n_left, self.n_right))
        out = np.empty((cap, 2), np.int32)
        n = C.c_int(0)
        _check(fn(self._h, *args, _ptr(out), cap, C.byref(n)), fn.__name__)
        return out[: n.value].copy()

    def find_putative_matches(self, min_score: float = 0.9, min_ratio: float = 0.8) -> np.ndarray:
        """SIFT_Matching::findPutativeMatches (v3d_cudamatching.h:45-46): (n, 2) (left, right)."""
        return self._result(lib().v3dm_putative, C.c_float(min_score), C.c_float(min_ratio))

    def run_guided_matching(self, F, distance_threshold: float, left_positions, right_positions,
                            min_score: float = 0.9, min_ratio: float = 0.8) -> np.ndarray:
        """SIFT_Matching::runGuidedMatching (v3d_cudamatching.h:48-52)."""
        Fm = np.ascontiguousarray(np.asarray(F, np.float64).reshape(3, 3))
        lp, rp = _pos(left_positions, self.n_left), _pos(right_positions, self.n_right)
        return self._result(lib().v3dm_guided_F, Fm.ctypes.data_as(C.POINTER(C.c_double)),
                            C.c_float(distance_threshold), _ptr(lp), _ptr(rp), C.c_float(min_score),
                            C.c_float(min_ratio))

    def run_guided_homography_matching(self, H, distance_threshold: float, left_positions, right_positions,
                                       min_score: float = 0.9, min_ratio: float = 0.8) -> np.ndarray:
        """SIFT_Matching::runGuidedHomographyMatching (v3d_cudamatching.h:54-58)."""
        Hm = np.ascontiguousarray(np.asarray(H, np.float64).reshape(3, 3))
        lp, rp = _pos(left_positions, self.n_left), _pos(right_positions, self.n_right)
        return self._result(lib().v3dm_guided_H, Hm.ctypes.data_as(C.POINTER(C.c_double)),
                            C.c_float(distance_threshold), _ptr(lp), _ptr(rp), C.c_float(min_score),
                            C.c_float(min_ratio))

    # ---- device-resident calls (pointers are device addresses, e.g. torch data_ptr()) ----
    def putative_device(self, min_score: float, min_ratio: float, d_pairs: int, d_count: int):
        _check(lib().v3dm_putative_device(self._h, min_score, min_ratio, C.c_void_p(d_pairs), C.c_void_p(d_count)),
               "putative_device")

    def guided_F_device(self, F, thr: float, d_lpos: int, d_rpos: int, min_score: float, min_ratio: float,
                        d_pairs: int, d_count: int):
        Fm = np.ascontiguousarray(np.asarray(F, np.float64).reshape(3, 3))
        _check(lib().v3dm_guided_F_device(self._h, Fm.ctypes.data_as(C.POINTER(C.c_double)), thr,
                                          C.c_void_p(d_lpos), C.c_void_p(d_rpos), min_score, min_ratio,
                                          C.c_void_p(d_pairs), C.c_void_p(d_count)), "guided_F_device")

    def wait(self) -> None:
        _check(lib().v3dm_matcher_wait(self._h), "wait")

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().v3dm_matcher_stream(self._h, C.byref(s)), "stream")
        return s.value or 0

    def num_configs(self) -> int:
        n = C.c_int(0)
        _check(lib().v3dm_matcher_num_configs(self._h, C.byref(n)), "num_configs")
        return n.value

    def config(self):
        """(config id, left rows per group, right columns per tile) of the fused kernel."""
        c, r, n = C.c_int(0), C.c_int(0), C.c_int(0)
        _check(lib().v3dm_matcher_get_config(self._h, C.byref(c), C.byref(r), C.byref(n)), "get_config")
        return c.value, r.value, n.value

    def set_config(self, cfg: int) -> None:
        _check(lib().v3dm_matcher_set_config(self._h, cfg), "set_config")

    def autotune(self, min_score: float = 0.9, min_ratio: float = 0.8, reps: int = 3):
        """Times every kernel configuration on the current features; keeps and returns the
        fastest as (config id, milliseconds per call)."""
        b, ms = C.c_int(0), C.c_double(0)
        _check(lib().v3dm_matcher_autotune(self._h, min_score, min_ratio, reps, C.byref(b), C.byref(ms)),
               "autotune")
        return b.value, ms.value

    def profile(self, enable: bool = True) -> None:
        _check(lib().v3dm_matcher_profile(self._h, int(enable)), "profile")

    def profile_read(self, pass_id: int | None = None):
        """(summed milliseconds, launches) of the fused matching kernel since profile():
        pass 0 = lefts x rights (the full contraction), pass 1 = chosen rights x lefts.
        Without pass_id: pass 0, clearing the record."""
        ms, n = C.c_double(0), C.c_int(0)
        if pass_id is None:
            _check(lib().v3dm_matcher_profile_read(self._h, C.byref(ms), C.byref(n)), "profile_read")
        else:
            _check(lib().v3dm_matcher_profile_read_pass(self._h, pass_id, C.byref(ms), C.byref(n)), "profile_read")
        return ms.value, n.value

    def test_wait_fault(self, wait_cycles: int, skip_load: int) -> None:
        """Failure-path test hook (v3dm_matcher_test_wait_fault): bounded waits of pass A give up
        after wait_cycles, and CTA 0 skips its skip_load-th tile load; (0, 0) turns it off."""
        _check(lib().v3dm_matcher_test_wait_fault(self._h, int(wait_cycles), int(skip_load)), "test_wait_fault")

    def last_launches(self) -> int:
        n = C.c_int(0)
        _check(lib().v3dm_matcher_last_launches(self._h, C.byref(n)), "last_launches")
        return n.value


def voctree_counts(branch_factor: int, depth: int):
    nc, lc = C.c_int64(0), C.c_int64(0)
    _check(lib().v3dm_voctree_counts(branch_factor, depth, C.byref(nc), C.byref(lc)), "voctree_counts")
    return nc.value, lc.value


class VocabularyTreeTraversal:
    """V3D_CUDA::VocabularyTreeTraversal<BranchFactor, Depth> with a runtime shape."""

    def __init__(self, branch_factor: int, depth: int, device: int = 0):
        h = C.c_void_p()
        _check(lib().v3dm_voctree_create(C.byref(h), device, branch_factor, depth), "VocabularyTreeTraversal()")
        self._h = h
        self.branch_factor, self.depth = branch_factor, depth

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.v3dm_voctree_destroy(self._h)
        self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def get_node_count(self) -> int:
        return voctree_counts(self.branch_factor, self.depth)[0]

    def get_leave_count(self) -> int:
        return voctree_counts(self.branch_factor, self.depth)[1]

    def allocate(self, n_max_features: int):
        _check(lib().v3dm_voctree_allocate(self._h, int(n_max_features)), "allocate")

    def set_nodes(self, nodes: np.ndarray):
        d = np.ascontiguousarray(nodes)
        if d.shape != (self.get_node_count(), 128):
            raise ValueError("nodes must be (node count, 128)")
        if d.dtype == np.uint8:
            _check(lib().v3dm_voctree_set_nodes_u8(self._h, _ptr(d)), "setNodes")
        else:
            d = np.ascontiguousarray(d, dtype=np.float32)
            _check(lib().v3dm_voctree_set_nodes_f32(self._h, _ptr(d)), "setNodes")

    def traverse_tree(self, features: np.ndarray, id_mode: int = LEAF_GLOBAL) -> np.ndarray:
        d, kind = _desc(features)
        out = np.empty(d.shape[0], np.int32)
        fn = lib().v3dm_voctree_quantize_u8 if kind == "u8" else lib().v3dm_voctree_quantize_f32
        _check(fn(self._h, d.shape[0], _ptr(d), _ptr(out), id_mode), "traverseTree")
        return out

    def quantize_device(self, n: int, d_keys: int, d_ids: int, id_mode: int = LEAF_GLOBAL):
        _check(lib().v3dm_voctree_quantize_u8_device(self._h, n, C.c_void_p(d_keys), C.c_void_p(d_ids), id_mode),
               "quantize_device")

    def quantize_f32_device(self, n: int, d_keys: int, d_ids: int, id_mode: int = LEAF_GLOBAL):
        """Float keys in device memory, the reference CPU tree's sequential FP32 order."""
        _check(lib().v3dm_voctree_quantize_f32_device(self._h, n, C.c_void_p(d_keys), C.c_void_p(d_ids), id_mode),
               "quantize_f32_device")

    def replays(self) -> int:
        """Key-levels decided by the sequential replay since the tree was created."""
        n = C.c_longlong(0)
        _check(lib().v3dm_voctree_replays(self._h, C.byref(n)), "replays")
        return n.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().v3dm_voctree_stream(self._h, C.byref(s)), "stream")
        return s.value or 0

    def last_launches(self) -> int:
        """Kernels launched by the last quantization call."""
        n = C.c_int32(0)
        _check(lib().v3dm_voctree_last_launches(self._h, C.byref(n)), "last_launches")
        return n.value


class BatchMatching:
    """Many image pairs matched together (the apps' per-pair findPutativeMatches loop,
    V3D/Apps/SfM/match_sequence.cpp:165-234).  Each pair's result equals
    SIFTMatching.find_putative_matches on the two images."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().v3dm_batch_create(C.byref(h), device), "batch_create")
        self._h = h
        self.n_pairs = 0

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.v3dm_batch_destroy(self._h)
        self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_images(self, desc: np.ndarray, counts) -> None:
        """desc: (sum(counts), 128) uint8 or float32, the images' descriptors concatenated.
        Float descriptors that are not all u/512 are matched as SIFTMatching matches them (the
        BF16 hi/lo scores); `float_mode` tells which layout was chosen."""
        c = np.ascontiguousarray(counts, dtype=np.int32)
        is_f = np.asarray(desc).dtype == np.float32
        d = np.ascontiguousarray(desc, dtype=np.float32 if is_f else np.uint8)
        if d.ndim != 2 or d.shape[1] != 128 or int(c.sum()) != d.shape[0]:
            raise ValueError("desc must be (sum(counts), 128) uint8 or float32")
        fn = lib().v3dm_batch_set_images_f32 if is_f else lib().v3dm_batch_set_images_u8
        _check(fn(self._h, c.shape[0], _ptr(c), _ptr(d)), "batch_set_images")

    def set_images_device(self, d_desc: int, counts, dtype=np.uint8) -> None:
        c = np.ascontiguousarray(counts, dtype=np.int32)
        fn = lib().v3dm_batch_set_images_f32_device if np.dtype(dtype) == np.float32 else \
            lib().v3dm_batch_set_images_u8_device
        _check(fn(self._h, c.shape[0], _ptr(c), C.c_void_p(d_desc)), "batch_set_images_device")

    @property
    def float_mode(self) -> bool:
        v = C.c_int(0)
        _check(lib().v3dm_batch_float_mode(self._h, C.byref(v)), "batch_float_mode")
        return bool(v.value)

    def set_pairs(self, pairs=None) -> None:
        """pairs: (n, 2) int32 (left image, right image); None = every (i, j), i < j."""
        if pairs is None:
            _check(lib().v3dm_batch_set_pairs(self._h, -1, None), "batch_set_pairs")
            n = C.c_longlong(0)
            ops = C.c_longlong(0)
            _check(lib().v3dm_batch_work(self._h, C.byref(ops), C.byref(n)), "batch_work")
            self.n_pairs = n.value
            return
        p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        _check(lib().v3dm_batch_set_pairs(self._h, p.shape[0], _ptr(p)), "batch_set_pairs")
        self.n_pairs = p.shape[0]

    def match(self, min_score: float = 0.9, min_ratio: float = 0.8, cap: int | None = None) -> np.ndarray:
        """(n, 3) int32 (pair index, left, right), grouped by pair, ascending left in a pair."""
        cap = cap if cap is not None else max(1 << 20, getattr(self, "_last_n", 0))
        while True:
            out = np.empty((max(1, cap), 3), np.int32)
            n = C.c_longlong(0)
            st = lib().v3dm_batch_match(self._h, min_score, min_ratio, _ptr(out), cap, C.byref(n))
            if st == ERR_CAPACITY:
                cap = n.value
                continue
            _check(st, "batch_match")
            self._last_n = n.value
            return out[: n.value].copy()

    def set_positions(self, positions: np.ndarray) -> None:
        """positions: (sum(counts), 2) float32, every descriptor's (x, y), in descriptor order."""
        p = np.ascontiguousarray(positions, dtype=np.float32)
        _check(lib().v3dm_batch_set_positions(self._h, _ptr(p)), "batch_set_positions")

    def match_guided(self, M: np.ndarray, thr, min_score: float = 0.9, min_ratio: float = 0.8,
                     homography: bool = False, cap: int | None = None) -> np.ndarray:
        """Guided matching of every pair (v3dm_batch_match_guided): M (n_pairs, 3, 3) fundamental
        matrices (or homographies), thr a threshold per pair (or one for all).  Triples like match()."""
        m = np.ascontiguousarray(M, dtype=np.float64).reshape(-1, 9)
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(thr, np.float32), (m.shape[0],)), dtype=np.float32)
        cap = cap if cap is not None else max(1 << 20, getattr(self, "_last_n", 0))
        while True:
            out = np.empty((max(1, cap), 3), np.int32)
            n = C.c_longlong(0)
            st = lib().v3dm_batch_match_guided(self._h, 2 if homography else 1, _ptr(m), _ptr(t), min_score,
                                               min_ratio, _ptr(out), cap, C.byref(n))
            if st == ERR_CAPACITY:
                cap = n.value
                continue
            _check(st, "batch_match_guided")
            self._last_n = n.value
            return out[: n.value].copy()

    def match_per_pair(self, min_score: float = 0.9, min_ratio: float = 0.8):
        """List with one (n, 2) (left, right) array per pair of the table."""
        return self.split_pairs(self.match(min_score, min_ratio))

    def split_pairs(self, t: np.ndarray):
        """(pair, left, right) triples -> one (n, 2) array per pair of the table."""
        order = np.argsort(t[:, 0], kind="stable")
        t = t[order]
        bounds = np.searchsorted(t[:, 0], np.arange(self.n_pairs + 1))
        return [t[bounds[k]:bounds[k + 1], 1:].copy() for k in range(self.n_pairs)]

    def match_proposal(self, projection, probes: int, min_score: float = 0.9, min_ratio: float = 0.8,
                       cap: int | None = None, probes_right: int = 1) -> np.ndarray:
        """Candidate-proposal matching (v3dm_batch_match_proposal): triples like match().
        probes: cells probed per left; probes_right: cells each right is listed under."""
        cap = cap if cap is not None else max(1 << 20, getattr(self, "_last_n", 0))
        while True:
            out = np.empty((max(1, cap), 3), np.int32)
            n = C.c_longlong(0)
            st = lib().v3dm_batch_match_proposal(self._h, projection.handle, probes, probes_right, min_score,
                                                 min_ratio, _ptr(out), cap, C.byref(n))
            if st == ERR_CAPACITY:
                cap = n.value
                continue
            _check(st, "batch_match_proposal")
            self._last_n = n.value
            return out[: n.value].copy()

    def match_proposal_device(self, projection, probes: int, min_score: float, min_ratio: float,
                              d_count: int = 0, probes_right: int = 1) -> None:
        _check(lib().v3dm_batch_match_proposal_device(self._h, projection.handle, probes, probes_right, min_score,
                                                      min_ratio, C.c_void_p(d_count) if d_count else None),
               "batch_match_proposal_device")

    def proposal_scored(self):
        """(pairs of descriptors the last proposal call scored, sum over pairs of nL * nR)."""
        a, b = C.c_longlong(0), C.c_longlong(0)
        _check(lib().v3dm_batch_proposal_scored(self._h, C.byref(a), C.byref(b)), "batch_proposal_scored")
        return a.value, b.value

    def match_device(self, min_score: float, min_ratio: float, d_count: int = 0) -> None:
        _check(lib().v3dm_batch_match_device(self._h, min_score, min_ratio, C.c_void_p(d_count) if d_count else None),
               "batch_match_device")

    def wait(self) -> int:
        """Checks the last device call; returns its status (ERR_CANDIDATES: repeat the call)."""
        st = lib().v3dm_batch_wait(self._h)
        if st not in (OK, ERR_CANDIDATES):
            _check(st, "batch_wait")
        return st

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().v3dm_batch_stream(self._h, C.byref(s)), "batch_stream")
        return s.value or 0

    def use_graph(self, enable: bool = True) -> None:
        _check(lib().v3dm_batch_use_graph(self._h, int(enable)), "batch_use_graph")

    def set_config(self, cfg: int, schedule: int = 0) -> None:
        _check(lib().v3dm_batch_set_config(self._h, cfg, schedule), "batch_set_config")

    def config(self):
        c, s = C.c_int(0), C.c_int(0)
        _check(lib().v3dm_batch_get_config(self._h, C.byref(c), C.byref(s)), "batch_get_config")
        return c.value, s.value

    def autotune(self, min_score: float = 0.9, min_ratio: float = 0.8, reps: int = 2):
        """Times every (configuration, schedule); keeps the fastest.  Returns (cfg, schedule,
        ms array indexed [cfg, schedule])."""
        c, s = C.c_int(0), C.c_int(0)
        ms = (C.c_float * 64)(*([-1.0] * 64))
        _check(lib().v3dm_batch_autotune(self._h, min_score, min_ratio, reps, C.byref(c), C.byref(s), ms),
               "batch_autotune")
        t = np.array(ms[:], np.float32)
        n = int(np.flatnonzero(t >= 0).max()) // 2 + 1
        return c.value, s.value, t[: 2 * n].reshape(n, 2)

    def profile(self, enable: bool = True) -> None:
        _check(lib().v3dm_batch_profile(self._h, int(enable)), "batch_profile")

    def profile_read(self, pass_id: int):
        ms, n = C.c_double(0), C.c_int(0)
        _check(lib().v3dm_batch_profile_read(self._h, pass_id, C.byref(ms), C.byref(n)), "batch_profile_read")
        return ms.value, n.value

    def last_launches(self) -> int:
        n = C.c_int(0)
        _check(lib().v3dm_batch_last_launches(self._h, C.byref(n)), "batch_last_launches")
        return n.value

    def work(self):
        """(int8 operations of the pair table, number of pairs)."""
        ops, n = C.c_longlong(0), C.c_longlong(0)
        _check(lib().v3dm_batch_work(self._h, C.byref(ops), C.byref(n)), "batch_work")
        return ops.value, n.value


PROJ_PARAMS = 10336
PROJ_MAX_CELLS = 256
PROJ_MAX_PROBES = 8
PROJ_MAX_BATCH = 4096


class Projection:
    """The learned 128 -> 64 -> 32 projection of the proposal matcher (v3dm_projection_*)."""

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        _check(lib().v3dm_projection_create(C.byref(h), device, seed), "projection_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.v3dm_projection_destroy(self._h)
        self._h = None

    __del__ = close

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def params(self) -> np.ndarray:
        out = np.empty(PROJ_PARAMS, np.float32)
        _check(lib().v3dm_projection_get_params(self._h, _ptr(out)), "projection_get_params")
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.shape != (PROJ_PARAMS,):
            raise ValueError(f"params must have {PROJ_PARAMS} entries")
        _check(lib().v3dm_projection_set_params(self._h, _ptr(p)), "projection_set_params")

    def loss_grad(self, anchors: np.ndarray, positives: np.ndarray, temperature: float):
        a = np.ascontiguousarray(anchors, np.uint8)
        p = np.ascontiguousarray(positives, np.uint8)
        g = np.empty(PROJ_PARAMS, np.float32)
        loss = C.c_float(0)
        _check(lib().v3dm_projection_loss_grad(self._h, _ptr(a), _ptr(p), a.shape[0], temperature, C.byref(loss),
                                               _ptr(g)), "projection_loss_grad")
        return loss.value, g

    def train_step(self, d_anchors: int, d_positives: int, batch: int, temperature: float, lr: float,
                   want_loss: bool = False):
        loss = C.c_float(0)
        _check(lib().v3dm_projection_train_step(self._h, C.c_void_p(d_anchors), C.c_void_p(d_positives), batch,
                                                temperature, lr, C.byref(loss) if want_loss else None),
               "projection_train_step")
        return loss.value if want_loss else None

    def embed(self, desc: np.ndarray) -> np.ndarray:
        d = np.ascontiguousarray(desc, np.uint8)
        z = np.empty((d.shape[0], 32), np.float32)
        _check(lib().v3dm_projection_embed(self._h, _ptr(d), d.shape[0], _ptr(z)), "projection_embed")
        return z

    def set_cells(self, centroids: np.ndarray) -> None:
        c = np.ascontiguousarray(centroids, np.float32)
        if c.ndim != 2 or c.shape[1] != 32:
            raise ValueError("centroids must be (C, 32)")
        _check(lib().v3dm_projection_set_cells(self._h, c.shape[0], _ptr(c)), "projection_set_cells")

    def assign(self, desc: np.ndarray, probes: int) -> np.ndarray:
        d = np.ascontiguousarray(desc, np.uint8)
        out = np.empty((d.shape[0], probes), np.uint8)
        _check(lib().v3dm_projection_assign(self._h, _ptr(d), d.shape[0], probes, _ptr(out)), "projection_assign")
        return out


# ---- feature files ----------------------------------------------------------------------------

LOAD_ROUND32 = 1
LOAD_KEEP_F32 = 2
LOAD_LOSSY_U8 = 4
ERR_IO = 11


def features_read(path: str) -> dict:
    """v3dm_features_read: the reference's feature archive (SerializableVector<SIFT_Feature>,
    binary "V3DBIN" or text "V3DTXT") as arrays: ids (n), positions (n, 2), directions (n, 2), scales (n), magnitudes (n),
    descriptors (n, 128) float32."""
    n = C.c_int32(0)
    p = str(path).encode()
    _check(lib().v3dm_features_read(p, 0, C.byref(n), None, None, None, None, None, None), "features_read")
    m = n.value
    out = {"ids": np.empty(m, np.int32), "positions": np.empty((m, 2), np.float32),
           "directions": np.empty((m, 2), np.float32), "scales": np.empty(m, np.float32),
           "magnitudes": np.empty(m, np.float32), "descriptors": np.empty((m, 128), np.float32)}
    _check(lib().v3dm_features_read(p, m, C.byref(n), *[_ptr(out[k]) for k in
                                                         ("ids", "positions", "directions", "scales",
                                                          "magnitudes", "descriptors")]), "features_read")
    return out


def quantize_u8_device(d_values: int, n_values: int, d_out: int, stream: int = 0) -> None:
    """v3dm_quantize_u8_device on device pointers (n_values a multiple of 4)."""
    _check(lib().v3dm_quantize_u8_device(C.c_void_p(d_values), C.c_longlong(n_values), C.c_void_p(d_out),
                                         C.c_void_p(stream)), "quantize_u8_device")


class Loader:
    """Feature-file loader (v3dm_loader_*): many files at once, descriptors copied to the device
    in one transfer.  They become u8 there when every value is u/512; the extractors' unit-L2
    floats are kept as floats with LOAD_KEEP_F32 (for the float matcher), refused by default
    (V3DMError NOT_U8), or rounded with LOAD_LOSSY_U8."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().v3dm_loader_create(device, C.byref(h)), "loader_create")
        self._h = h

    def close(self) -> None:
        if self._h:
            lib().v3dm_loader_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def load(self, paths, max_per_image: int = 0, flags: int = 0) -> np.ndarray:
        """Reads the files; returns the kept feature count of each."""
        arr = (C.c_char_p * len(paths))(*[str(p).encode() for p in paths])
        counts = np.zeros(len(paths), np.int32)
        _check(lib().v3dm_loader_load(self._h, len(paths), arr, max_per_image, flags, _ptr(counts)), "loader_load")
        return counts

    def descriptors_device(self):
        """(device pointer of the u8 descriptors, their count)."""
        p, n = C.c_void_p(), C.c_longlong(0)
        _check(lib().v3dm_loader_descriptors_device(self._h, C.byref(p), C.byref(n)), "loader_descriptors_device")
        return p.value or 0, n.value

    def descriptors_f32_device(self):
        """(device pointer of the float descriptors, their count); after a LOAD_KEEP_F32 load."""
        p, n = C.c_void_p(), C.c_longlong(0)
        _check(lib().v3dm_loader_descriptors_f32_device(self._h, C.byref(p), C.byref(n)),
               "loader_descriptors_f32_device")
        return p.value or 0, n.value

    def exact_u8(self) -> bool:
        """True when every descriptor value of the last load was exactly u/512."""
        e = C.c_int(0)
        _check(lib().v3dm_loader_exact_u8(self._h, C.byref(e)), "loader_exact_u8")
        return bool(e.value)

    def positions(self) -> np.ndarray:
        p, n = C.c_void_p(), C.c_longlong(0)
        lib().v3dm_loader_descriptors_device(self._h, C.byref(p), C.byref(n))  # the count, whatever the status
        out = np.empty((n.value, 2), np.float32)
        _check(lib().v3dm_loader_positions(self._h, _ptr(out)), "loader_positions")
        return out


RETRIEVAL_MAX_IMAGES = 32768
RETRIEVAL_MAX_BEST = 1024


def _offsets_words(offsets, words):
    off = np.ascontiguousarray(offsets, np.int32)
    w = np.ascontiguousarray(words, np.int32)
    if off.ndim != 1 or off.shape[0] < 1 or (off.shape[0] > 1 and off[-1] > w.shape[0]):
        raise ValueError("offsets must hold nImages + 1 entries, the last one <= len(words)")
    return off, w


class Retrieval:
    """Retrieval scoring of a whole image sequence (v3dm_retrieval_*): the voctree app's image
    loop over LeafDocuments::computeBinomialScores / insertDocument
    (match_using_voctree.cpp:176-222, V3D/Base/v3d_voctree.h:143-278) in one call."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().v3dm_retrieval_create(C.byref(h), device), "retrieval_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.v3dm_retrieval_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def binomial(self, n_leaves: int, offsets, words, p_match: float = 0.1, n_best: int = 20):
        """(best_docs, best_scores), nImages x n_best: row i = the min(n_best, i) best earlier
        images of image i, best first, then -1 / 0."""
        off, w = _offsets_words(offsets, words)
        n = off.shape[0] - 1
        docs = np.empty((n, n_best), np.int32)
        sc = np.empty((n, n_best), np.float32)
        _check(lib().v3dm_retrieval_binomial(self._h, n_leaves, n, _ptr(off), _ptr(w), float(p_match), n_best,
                                             _ptr(docs), _ptr(sc)), "retrieval_binomial")
        return docs, sc

    def binomial_device(self, n_leaves: int, offsets, d_words: int, p_match: float, n_best: int, d_docs: int,
                        d_scores: int) -> None:
        off = np.ascontiguousarray(offsets, np.int32)
        _check(lib().v3dm_retrieval_binomial_device(self._h, n_leaves, off.shape[0] - 1, _ptr(off),
                                                    C.c_void_p(d_words), float(p_match), n_best,
                                                    C.c_void_p(d_docs), C.c_void_p(d_scores)),
               "retrieval_binomial_device")

    def wait(self) -> None:
        _check(lib().v3dm_retrieval_wait(self._h), "retrieval_wait")

    def profile(self, enable: bool = True) -> None:
        _check(lib().v3dm_retrieval_profile(self._h, int(enable)), "retrieval_profile")

    def profile_read(self, kernel: int):
        """(milliseconds, launches) of kernel 0 (bitmap) or 1 (scores) since the last read."""
        ms, n = C.c_double(0.0), C.c_int(0)
        _check(lib().v3dm_retrieval_profile_read(self._h, kernel, C.byref(ms), C.byref(n)), "retrieval_profile_read")
        return ms.value, n.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().v3dm_retrieval_stream(self._h, C.byref(s)), "retrieval_stream")
        return s.value or 0


def retrieval_pairs(best_docs: np.ndarray) -> np.ndarray:
    """The app's putativePairwiseMatches as (view1, view2) pairs, view1 the retrieved earlier
    image, ordered by view1 then view2 (v3dm_retrieval_pairs): the pair table of
    BatchMatching.set_pairs."""
    d = np.ascontiguousarray(best_docs, np.int32)
    n, k = (d.shape[0], d.shape[1]) if d.ndim == 2 else (0, 1)
    cnt = C.c_longlong(0)
    _check(lib().v3dm_retrieval_pairs(n, k, _ptr(d), 0, None, C.byref(cnt)), "retrieval_pairs")
    out = np.empty((cnt.value, 2), np.int32)
    _check(lib().v3dm_retrieval_pairs(n, k, _ptr(d), cnt.value, _ptr(out), C.byref(cnt)), "retrieval_pairs")
    return out


class LeafDocuments:
    """V3D::LeafDocuments (v3d_voctree.h:105-289) for code written against its incremental
    interface: insert_document(words) and compute_binomial_scores(p_match, words, n_best).
    Each query runs the whole-sequence scoring of Retrieval on the inserted documents plus the
    query and keeps the last row; the batched Retrieval.binomial is the fast path."""

    def __init__(self, n_leaves: int, device: int = 0):
        self.n_leaves = int(n_leaves)
        self._docs: list[np.ndarray] = []
        self._r = Retrieval(device)

    def insert_document(self, visual_words) -> int:
        """Returns the document id (0, 1, ... in insertion order)."""
        w = np.ascontiguousarray(visual_words, np.int32)
        if w.size and (w.min() < 0 or w.max() >= self.n_leaves):
            raise V3DMError(ERR_ARG, "insertDocument")
        self._docs.append(w)
        return len(self._docs) - 1

    def compute_binomial_scores(self, p_match: float, visual_words, n_best: int = -1):
        """[(score, document id)] ascending, the n_best best (every document when n_best < 0)."""
        nd = len(self._docs)
        k = nd if n_best < 0 or n_best > nd else n_best
        if nd == 0 or k == 0:
            return []
        parts = self._docs + [np.ascontiguousarray(visual_words, np.int32)]
        off = np.zeros(nd + 2, np.int32)
        off[1:] = np.cumsum([p.shape[0] for p in parts])
        docs, sc = self._r.binomial(self.n_leaves, off, np.concatenate(parts), p_match, k)
        return [(float(sc[nd, j]), int(docs[nd, j])) for j in range(k)]


RANSAC_MAX_DRAW = 65536
RANSAC_MAX_SAMPLES = 4194304
RANSAC_MAX_PAIRS = 32768


def ransac_shuffle_samples(n: int, n_samples: int, seed: int) -> np.ndarray:
    """The 5-correspondence samples computeRobustOrientationMLE draws after srand(seed), in loop
    order ((k, 5) int32, at most n_samples + 1 rows)."""
    cap = n_samples + 1
    out = np.empty((cap, 5), np.int32)
    nd = C.c_int(0)
    _check(lib().v3dm_ransac_shuffle_samples(int(n), int(n_samples), int(seed) & 0xffffffff, cap, _ptr(out),
                                             C.byref(nd)), "ransac_shuffle_samples")
    return out[:nd.value].copy()


class Ransac:
    """computeRobustOrientationMLE (reconstruction_common.cpp:139-340, no iterative refinement)
    for many pairs at once (v3dm_ransac_essential)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().v3dm_ransac_create(C.byref(h), device), "ransac_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.v3dm_ransac_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_refinement(self, enable: bool) -> None:
        """RobustOrientationMode::iterativeRefinement (the apps switch it on)."""
        _check(lib().v3dm_ransac_set_refinement(self._h, int(bool(enable))), "ransac_set_refinement")

    def essential(self, offsets, corrs, K, inlier_threshold: float, n_samples: int = 1000, samples=None,
                  n_draw: int | None = None, seed: int = 0, flags: bool = True):
        """offsets (nPairs + 1), corrs (N, 4) float32 pixel positions (left x, y, right x, y), K
        (nPairs, 2, 3, 3); samples (nPairs, nDraw, 5) int32 or None (drawn on the device).
        Returns dict(models (nPairs, 31), E, F, R, T, error, n_inliers, flags)."""
        off = np.ascontiguousarray(offsets, np.int32)
        n_pairs = off.shape[0] - 1
        c = np.ascontiguousarray(corrs, np.float32).reshape(-1, 4)
        k = np.ascontiguousarray(K, np.float64).reshape(n_pairs, 18)
        if samples is not None:
            smp = np.ascontiguousarray(samples, np.int32)
            n_draw = smp.shape[1]
            sp = _ptr(smp)
        else:
            n_draw = n_samples + 1 if n_draw is None else n_draw
            sp = None
        models = np.empty((n_pairs, 31), np.float64)
        nin = np.empty(n_pairs, np.int32)
        fl = np.empty(c.shape[0], np.uint8) if flags else None
        _check(lib().v3dm_ransac_essential(self._h, n_pairs, _ptr(off), _ptr(c), _ptr(k), float(inlier_threshold),
                                           int(n_samples), int(n_draw), sp, int(seed) & 0xffffffffffffffff,
                                           _ptr(models), _ptr(nin), _ptr(fl) if fl is not None else None),
               "ransac_essential")
        return {"models": models, "E": models[:, :9].reshape(-1, 3, 3), "F": models[:, 9:18].reshape(-1, 3, 3),
                "R": models[:, 18:27].reshape(-1, 3, 3), "T": models[:, 27:30], "error": models[:, 30],
                "n_inliers": nin, "flags": fl}

    def essential_device(self, offsets, d_corrs: int, K, inlier_threshold: float, n_samples: int, n_draw: int,
                         d_samples: int | None, seed: int, d_models: int, d_n_inliers: int, d_flags: int) -> None:
        off = np.ascontiguousarray(offsets, np.int32)
        n_pairs = off.shape[0] - 1
        k = np.ascontiguousarray(K, np.float64).reshape(n_pairs, 18)
        _check(lib().v3dm_ransac_essential_device(self._h, n_pairs, _ptr(off), C.c_void_p(d_corrs), _ptr(k),
                                                  float(inlier_threshold), int(n_samples), int(n_draw),
                                                  C.c_void_p(d_samples) if d_samples else None,
                                                  int(seed) & 0xffffffffffffffff, C.c_void_p(d_models),
                                                  C.c_void_p(d_n_inliers), C.c_void_p(d_flags)),
               "ransac_essential_device")

    def wait(self) -> None:
        _check(lib().v3dm_ransac_wait(self._h), "ransac_wait")

    def profile(self, enable: bool = True) -> None:
        _check(lib().v3dm_ransac_profile(self._h, int(enable)), "ransac_profile")

    def candidates(self):
        """(candidates scored, Sampson evaluations) of the last call."""
        a, b = C.c_longlong(0), C.c_longlong(0)
        _check(lib().v3dm_ransac_candidates(self._h, C.byref(a), C.byref(b)), "ransac_candidates")
        return a.value, b.value

    def profile_read(self, kernel: int):
        """(milliseconds, launches) of kernel 0 (five-point) or 1 (costs) since the last read."""
        ms, n = C.c_double(0.0), C.c_int(0)
        _check(lib().v3dm_ransac_profile_read(self._h, kernel, C.byref(ms), C.byref(n)), "ransac_profile_read")
        return ms.value, n.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().v3dm_ransac_stream(self._h, C.byref(s)), "ransac_stream")
        return s.value or 0

    def five_point(self, pts: np.ndarray):
        """Solutions of (n, 20) samples (x1[5] y1[5] x2[5] y2[5]): (Es (n, 10, 3, 3), counts)."""
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 20)
        es = np.zeros((p.shape[0], 10, 3, 3), np.float64)
        cnt = np.empty(p.shape[0], np.int32)
        _check(lib().v3dm_essential_five_point(self._h, p.shape[0], _ptr(p), _ptr(es), _ptr(cnt)), "five_point")
        return es, cnt

    def last_launches(self) -> int:
        n = C.c_int(0)
        _check(lib().v3dm_ransac_last_launches(self._h, C.byref(n)), "ransac_last_launches")
        return n.value
