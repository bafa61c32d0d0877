"""Seeded synthetic workloads for the matching path (no dataset ships with the reference).

The shapes and value distributions follow the five benchmark workloads of this project:

* ``pair``       one image pair, 4096 x 4096 SIFT-like uint8 descriptors, 30% of the right
                 set are noisy copies of random left descriptors;
* ``stereo``     one 16384 x 16384 pair whose planted matches obey a fundamental matrix of a
                 random stereo rig (for guided matching);
* ``images``     many images with uneven feature counts and shared feature tracks (batched
                 all-pairs matching);
* ``voctree``    a hierarchical k-means vocabulary tree and query descriptors;
* ``sequence_words``  the visual words of an image sequence (retrieval scoring);
* ``two_view_pairs``  putative correspondences of many image pairs (essential-matrix RANSAC).

Descriptor generator: i.i.d. Gamma(k=0.6, theta=1) components, L2-normalised, clamped at
0.2, renormalised, scaled by 512, rounded and clamped to 0..255 (the SIFT normalisation of
V3D/Base/v3d_feature.h:19-39 followed by the uint8 quantisation u = 512 * f).
"""
from __future__ import annotations

import numpy as np

MIN_SCORE = 0.7
MIN_RATIO = 0.8


def rng_for(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def sift_like(rng: np.random.Generator, n: int) -> np.ndarray:
    """n x 128 uint8 SIFT-like descriptors."""
    out = np.empty((n, 128), np.uint8)
    step = 1 << 18
    for s in range(0, n, step):
        e = min(n, s + step)
        x = rng.gamma(0.6, 1.0, size=(e - s, 128)).astype(np.float32)
        x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
        np.minimum(x, 0.2, out=x)
        x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
        out[s:e] = np.clip(np.rint(x * 512.0), 0, 255).astype(np.uint8)
    return out


def noisy_copy(rng: np.random.Generator, u: np.ndarray, sigma: float = 8.0) -> np.ndarray:
    """Copies of uint8 descriptors with N(0, sigma^2) noise, re-rounded and clamped."""
    v = u.astype(np.float32) + rng.normal(0.0, sigma, size=u.shape).astype(np.float32)
    return np.clip(np.rint(v), 0, 255).astype(np.uint8)


def pair(seed: int = 0, n_left: int = 4096, n_right: int = 4096, planted: float = 0.3):
    """One image pair.  Returns (L, R, truth) with truth[r] = planted left index or -1."""
    rng = rng_for(seed)
    L = sift_like(rng, n_left)
    n_p = int(round(planted * n_right)) if n_left > 0 else 0
    src = rng.integers(0, n_left, n_p)
    R = np.concatenate([noisy_copy(rng, L[src]), sift_like(rng, n_right - n_p)])
    truth = np.concatenate([src, -np.ones(n_right - n_p, np.int64)])
    perm = rng.permutation(n_right)
    return L, R[perm].copy(), truth[perm].copy()


def rig(rng: np.random.Generator, f: float = 1200.0, width: int = 1600, height: int = 1200,
        baseline: float = 0.3, max_yaw_deg: float = 10.0):
    """Random stereo rig.  Returns (K, Rot, t, F) with X2 = Rot X1 + t and q^T F p = 0."""
    K = np.array([[f, 0, width / 2.0], [0, f, height / 2.0], [0, 0, 1.0]])
    yaw = np.deg2rad(rng.uniform(-max_yaw_deg, max_yaw_deg))
    c, s = np.cos(yaw), np.sin(yaw)
    Rot = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    C2 = np.array([baseline, 0.0, 0.0])
    t = -Rot @ C2
    tx = np.array([[0, -t[2], t[1]], [t[2], 0, -t[0]], [-t[1], t[0], 0]])
    Ki = np.linalg.inv(K)
    F = Ki.T @ tx @ Rot @ Ki
    return K, Rot, t, F


def stereo(seed: int = 1, n_left: int = 16384, n_right: int = 16384, planted: float = 0.3,
           width: int = 1600, height: int = 1200, noise_px: float = 1.0):
    """Guided-matching pair: (L, R, lpos, rpos, F, truth).  Planted right features are the
    projections of the 3-D point behind a left keypoint (depth U(2, 20) m) plus N(0, 1 px)
    noise, with noisy-copy descriptors; the rest are fresh features at uniform positions."""
    rng = rng_for(seed)
    K, Rot, t, F = rig(rng, width=width, height=height)
    L = sift_like(rng, n_left)
    lpos = np.stack([rng.uniform(0, width, n_left), rng.uniform(0, height, n_left)], 1)
    n_p = min(int(round(planted * n_right)), n_left)
    src = rng.choice(n_left, n_p, replace=False)
    depth = rng.uniform(2.0, 20.0, n_p)
    rays = np.linalg.inv(K) @ np.vstack([lpos[src].T, np.ones(n_p)])
    X1 = rays * depth
    X2 = Rot @ X1 + t[:, None]
    q = K @ X2
    qpos = (q[:2] / q[2]).T + rng.normal(0.0, noise_px, (n_p, 2))
    R = np.concatenate([noisy_copy(rng, L[src]), sift_like(rng, n_right - n_p)])
    rpos = np.concatenate([qpos, np.stack([rng.uniform(0, width, n_right - n_p),
                                           rng.uniform(0, height, n_right - n_p)], 1)])
    truth = np.concatenate([src, -np.ones(n_right - n_p, np.int64)])
    perm = rng.permutation(n_right)
    return (L, R[perm].copy(), lpos.astype(np.float32), rpos[perm].astype(np.float32), F,
            truth[perm].copy())


def images(seed: int = 2, n_images: int = 200, n_min: int = 1000, n_max: int = 12000,
           track_frac: float = 0.15, track_len=(2, 8), tracks: bool = False):
    """Image set for all-pairs matching.  Returns (desc, counts, offsets): desc is the
    concatenation of all images' uint8 descriptors.  A track is a base descriptor observed
    in a random subset of images with per-view N(0, 8^2) noise; track observations make up
    track_frac of every image's features.  With tracks=True a fourth array gives every
    descriptor's track id (-1: an unrelated descriptor); the descriptors are the same."""
    rng = rng_for(seed)
    counts = rng.integers(n_min, n_max + 1, n_images)
    slots = np.rint(track_frac * counts).astype(np.int64)
    remaining = slots.copy()
    obs_img, obs_track = [], []
    n_tracks = 0
    while True:
        avail = np.flatnonzero(remaining > 0)
        if avail.size < 2:
            break
        k = min(int(rng.integers(track_len[0], track_len[1] + 1)), avail.size)
        p = remaining[avail] / remaining[avail].sum()
        members = rng.choice(avail, k, replace=False, p=p)
        remaining[members] -= 1
        obs_img.append(members)
        obs_track.append(np.full(k, n_tracks))
        n_tracks += 1
    obs_img = np.concatenate(obs_img) if obs_img else np.zeros(0, np.int64)
    obs_track = np.concatenate(obs_track) if obs_track else np.zeros(0, np.int64)
    base = sift_like(rng, n_tracks)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    desc = np.empty((int(offsets[-1]), 128), np.uint8)
    order = np.argsort(obs_img, kind="stable")
    obs_img, obs_track = obs_img[order], obs_track[order]
    starts = np.searchsorted(obs_img, np.arange(n_images))
    ends = np.searchsorted(obs_img, np.arange(n_images), side="right")
    track_id = np.full(int(offsets[-1]), -1, np.int64)
    for i in range(n_images):
        tr = obs_track[starts[i]:ends[i]]
        feats = np.concatenate([noisy_copy(rng, base[tr]), sift_like(rng, int(counts[i]) - tr.size)])
        perm = rng.permutation(int(counts[i]))
        desc[offsets[i]:offsets[i + 1]] = feats[perm]
        track_id[offsets[i]:offsets[i + 1]] = np.concatenate([tr, np.full(int(counts[i]) - tr.size, -1)])[perm]
    if tracks:
        return desc, counts.astype(np.int32), offsets, track_id
    return desc, counts.astype(np.int32), offsets


def scene(seed: int = 6, n_images: int = 12, n_min: int = 500, n_max: int = 4000, track_frac: float = 0.3,
          f: float = 1200.0, width: int = 1600, height: int = 1200, spacing: float = 0.3,
          max_yaw_deg: float = 10.0, noise_px: float = 1.0):
    """An image set with geometry for guided matching.  The descriptors and tracks are those of
    images(seed, ...); image c is a camera at (spacing * c, 0, 0) with a random yaw, every track
    is a 3-D point in front of the cameras, and a track observation sits at the point's
    projection plus N(0, noise_px^2) noise; other features are uniform in the image.  Returns
    (desc, counts, offsets, positions (n, 2) float32, cams) with cams = (K, rotations, centres)."""
    desc, counts, offsets, track_id = images(seed, n_images, n_min, n_max, track_frac, tracks=True)
    rng = rng_for(seed + 1000)
    K = np.array([[f, 0, width / 2.0], [0, f, height / 2.0], [0, 0, 1.0]])
    rots, centres = [], []
    for c in range(n_images):
        yaw = np.deg2rad(rng.uniform(-max_yaw_deg, max_yaw_deg))
        co, si = np.cos(yaw), np.sin(yaw)
        rots.append(np.array([[co, 0, si], [0, 1, 0], [-si, 0, co]]))
        centres.append(np.array([spacing * c, 0.0, 0.0]))
    n_tracks = int(track_id.max()) + 1 if track_id.size else 0
    X = np.stack([rng.uniform(-6.0, 6.0 + spacing * n_images, n_tracks), rng.uniform(-4.0, 4.0, n_tracks),
                  rng.uniform(4.0, 20.0, n_tracks)], 1)
    pos = np.stack([rng.uniform(0, width, desc.shape[0]), rng.uniform(0, height, desc.shape[0])], 1)
    for c in range(n_images):
        sl = slice(int(offsets[c]), int(offsets[c + 1]))
        tr = track_id[sl]
        m = tr >= 0
        Xc = (rots[c] @ (X[tr[m]] - centres[c]).T)
        q = K @ Xc
        p = pos[sl]
        p[m] = (q[:2] / q[2]).T + rng.normal(0.0, noise_px, (int(m.sum()), 2))
    return desc, counts, offsets, pos.astype(np.float32), (K, rots, centres)


def float_from_u8(desc: np.ndarray, seed: int, sigma: float = 0.004) -> np.ndarray:
    """Float descriptors that are not u/512: desc / 512 perturbed by |N(0, sigma^2)| noise and
    renormalised to unit length (the values SIFT pipelines that keep floats hand over)."""
    rng = rng_for(2000 + seed)
    x = desc.astype(np.float64) / 512.0
    y = np.abs(x + rng.normal(0.0, sigma, x.shape))
    y /= np.maximum(np.linalg.norm(y, axis=1, keepdims=True), 1e-12)
    return y.astype(np.float32)


def fundamental(cams, i: int, j: int) -> np.ndarray:
    """F with q^T F p = 0 for p in image i and q in image j of a scene()."""
    K, rots, centres = cams
    Rot = rots[j] @ rots[i].T
    t = rots[j] @ (centres[i] - centres[j])
    tx = np.array([[0, -t[2], t[1]], [t[2], 0, -t[0]], [-t[1], t[0], 0]])
    Ki = np.linalg.inv(K)
    return Ki.T @ tx @ Rot @ Ki


def inlier_mask(triples: np.ndarray, pairs: np.ndarray, offsets: np.ndarray, track_id: np.ndarray) -> np.ndarray:
    """True for the match triples (pair, left, right) that join two views of one track."""
    tl = track_id[offsets[pairs[triples[:, 0], 0]] + triples[:, 1]]
    tr = track_id[offsets[pairs[triples[:, 0], 1]] + triples[:, 2]]
    return (tl >= 0) & (tl == tr)


def all_pairs(n_images: int) -> np.ndarray:
    """All unordered pairs (i, j), i < j, left = i."""
    i, j = np.triu_indices(n_images, 1)
    return np.stack([i, j], 1).astype(np.int32)


def unit_sift(rng: np.random.Generator, n: int) -> np.ndarray:
    """n x 128 float32 SIFT-like descriptors as the extractors store them: Gamma(0.6) values,
    L2-normalised, clamped at 0.2 and normalised again (SIFT_Feature::normalizeDescriptor after
    the extractor's clamp); not of the form u/512."""
    out = np.empty((n, 128), np.float32)
    step = 1 << 18
    for s in range(0, n, step):
        e = min(n, s + step)
        x = rng.gamma(0.6, 1.0, size=(e - s, 128)).astype(np.float32)
        x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
        np.minimum(x, 0.2, out=x)
        x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
        out[s:e] = x
    return out


def hkm_tree(rng: np.random.Generator, data: np.ndarray, bf: int, depth: int, iters: int = 4,
             chunk: int = 1 << 16) -> np.ndarray:
    """Hierarchical k-means vocabulary tree.

    Returns nodeCount x 128 centres in breadth-first order without the root (the layout of
    V3D/Base/v3d_voctree.h:22-34): uint8 rounded means for uint8 data, float32 means for float
    data (the apps' trees: k-means centres of unit-L2 descriptors).  Points are assigned to the
    child with the largest dot product, the rule the quantizer descends by.  A cluster that
    loses all its points keeps its previous centre; a node with fewer points than children seeds
    the missing children from noisy copies of its points (or fresh descriptors)."""
    floats = data.dtype != np.uint8
    n = data.shape[0]
    node_of = np.zeros(n, np.int64)  # node index (global, -1 = root) of each point's current node
    level_nodes = 1
    out = []
    parent_base = -1
    for d in range(depth):
        n_parents = level_nodes
        # group points by parent (local parent index 0..n_parents-1)
        local_parent = node_of - (parent_base if d > 0 else 0) if d > 0 else np.zeros(n, np.int64)
        order = np.argsort(local_parent, kind="stable")
        sp = local_parent[order]
        starts = np.searchsorted(sp, np.arange(n_parents))
        cnt = np.searchsorted(sp, np.arange(n_parents), side="right") - starts
        # init: bf random members per parent (with replacement), noisy so duplicates split
        pick = starts[:, None] + (rng.random((n_parents, bf)) * np.maximum(cnt, 1)[:, None]).astype(np.int64)
        pick = np.minimum(pick, n - 1)
        cent = data[order[pick.reshape(-1)]].reshape(n_parents, bf, 128)
        if floats:
            cent = np.abs(cent + rng.normal(0.0, 4.0 / 512, size=cent.shape)).astype(np.float32)
        else:
            cent = noisy_copy(rng, cent, 4.0)
        empty = cnt == 0
        if empty.any():
            fresh = unit_sift if floats else sift_like
            cent[empty] = fresh(rng, int(empty.sum()) * bf).reshape(-1, bf, 128)
        centf = cent.astype(np.float32)
        for it in range(iters + 1):
            child = np.empty(n, np.int64)
            for s in range(0, n, chunk):
                e = min(n, s + chunk)
                c = centf[local_parent[s:e]]  # (m, bf, 128)
                scores = np.einsum("mkd,md->mk", c, data[s:e].astype(np.float32))
                child[s:e] = np.argmax(scores, axis=1)  # first max on ties
            if it == iters:
                break
            idx = local_parent * bf + child
            sums = np.zeros((n_parents * bf, 128), np.float64)
            _segment_sum(sums, idx, data)
            num = np.bincount(idx, minlength=n_parents * bf)
            has = num > 0
            newc = centf.reshape(-1, 128).copy()
            if floats:
                newc[has] = sums[has] / num[has, None]
            else:
                newc[has] = np.clip(np.rint(sums[has] / num[has, None]), 0, 255)
            centf = newc.reshape(n_parents, bf, 128).astype(np.float32)
        out.append((centf if floats else centf.astype(np.uint8)).reshape(-1, 128))
        level_start = sum(bf ** (k + 1) for k in range(d))
        node_of = level_start + local_parent * bf + child
        parent_base = level_start
        level_nodes = n_parents * bf
    return np.concatenate(out, 0)


def _segment_sum(sums: np.ndarray, idx: np.ndarray, data: np.ndarray) -> None:
    """sums[k] = sum of data rows with idx == k."""
    order = np.argsort(idx, kind="stable")
    uniq, first = np.unique(idx[order], return_index=True)
    sums[uniq] = np.add.reduceat(data[order].astype(np.float64), first, axis=0)


def voctree(seed: int = 3, bf: int = 10, depth: int = 6, n_train: int = 500_000,
            n_query: int = 2_000_000, iters: int = 4, floats: bool = False):
    """(nodes, queries): an HKM tree trained on n_train descriptors and n_query queries; uint8
    (u/512) data, or with floats=True unit-L2 float descriptors and float k-means centres."""
    rng = rng_for(seed)
    gen = unit_sift if floats else sift_like
    train = gen(rng, n_train)
    nodes = hkm_tree(rng, train, bf, depth, iters)
    queries = gen(rng, n_query)
    return nodes, queries


def feature_arrays(rng: np.random.Generator, n: int, desc_u8: np.ndarray | None = None) -> dict:
    """Arrays of n SIFT_Feature records: ids, positions (n, 2) in a 1600 x 1200 image,
    directions, scales, magnitudes and float descriptors (u/512 of SIFT-like u8 when desc_u8 is
    None)."""
    if desc_u8 is None:
        desc_u8 = sift_like(rng, n)
    ang = rng.uniform(-np.pi, np.pi, n)
    return {"ids": np.arange(n, dtype=np.int32),
            "positions": np.stack([rng.uniform(0, 1600, n), rng.uniform(0, 1200, n)], 1).astype(np.float32),
            "directions": np.stack([np.cos(ang), np.sin(ang)], 1).astype(np.float32),
            "scales": rng.uniform(1.0, 12.0, n).astype(np.float32),
            "magnitudes": rng.uniform(0.0, 1.0, n).astype(np.float32),
            "descriptors": (desc_u8.astype(np.float32) / 512.0).astype(np.float32)}


def write_features(path, f: dict) -> None:
    """The reference's binary feature archive of f (the layout serializeDataToFile writes for a
    SerializableVector<SIFT_Feature>): "V3DBIN", uint32 count, then per feature int32 id and 134
    little-endian floats."""
    n = f["ids"].shape[0]
    rec = np.zeros(n, dtype=np.dtype([("id", "<i4"), ("six", "<f4", (6,)), ("desc", "<f4", (128,))]))
    rec["id"] = f["ids"]
    rec["six"] = np.concatenate([f["positions"], f["directions"], f["scales"][:, None], f["magnitudes"][:, None]], 1)
    rec["desc"] = f["descriptors"]
    with open(path, "wb") as fh:
        fh.write(b"V3DBIN")
        fh.write(np.uint32(n).astype("<u4").tobytes())
        fh.write(rec.tobytes())


def write_features_text(path, f: dict) -> None:
    """The reference's text feature archive of f (serializeDataToFile(..., writeBinary = false)):
    "V3DTXT", then the tokens TextOStreamArchive writes, each followed by a blank: the count, "{",
    per feature "SIFT_Feature", "{", the id and 134 values printed with 6 significant digits (the
    stream's default precision) and "}" with a line break and the 2-blank indentation, then "}"
    and a line break."""
    n = f["ids"].shape[0]
    six = np.concatenate([f["positions"], f["directions"], f["scales"][:, None], f["magnitudes"][:, None]], 1)
    parts = [f"V3DTXT\n{n} {{ "]
    for i in range(n):
        vals = " ".join(f"{float(v):g}" for v in (*six[i], *f["descriptors"][i]))
        parts.append(f"SIFT_Feature {{ {int(f['ids'][i])} {vals} }} \n  ")
    parts.append("} \n")
    with open(path, "w") as fh:
        fh.write("".join(parts))


def sequence_words(seed: int = 4, n_images: int = 2048, n_leaves: int = 125_000, n_min: int = 2000,
                   n_max: int = 6000, window: int = 8, keep: float = 0.6, zipf: float = 0.5):
    """Visual words of an image sequence: a scene of points, each with a word drawn from a Zipf
    law over the leaves (popular leaves are shared by many unrelated points; exponent 0.5: the
    most frequent of 125,000 leaves holds 0.14% of the words, about 180 times the mean); image i
    sees the points of a window that slides by 1/window of its width per image, each with
    probability 'keep', plus random background words.  Images within a few indices of each other share
    words.  Returns (offsets, words) with offsets[n_images + 1], words int32 in 0..n_leaves-1."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(n_min, n_max + 1, n_images)
    per_view = int(np.mean(counts) / keep * 0.7)  # points in a window
    step = max(1, per_view // window)
    n_points = step * (n_images - 1) + per_view
    rank = np.arange(1, n_leaves + 1, dtype=np.float64) ** -zipf
    cdf = np.cumsum(rank / rank.sum())
    perm = rng.permutation(n_leaves).astype(np.int32)  # popular leaves spread over the tree

    def zipf_words(n):
        return perm[np.minimum(np.searchsorted(cdf, rng.random(n)), n_leaves - 1)]

    point_word = zipf_words(n_points)
    parts = []
    for i in range(n_images):
        seen = point_word[i * step:i * step + per_view]
        seen = seen[rng.random(seen.shape[0]) < keep]
        n = int(counts[i])
        if seen.shape[0] >= n:
            w = seen[rng.permutation(seen.shape[0])[:n]]
        else:
            w = np.concatenate([seen, zipf_words(n - seen.shape[0])])
        parts.append(w[rng.permutation(n)].astype(np.int32))
    offsets = np.zeros(n_images + 1, np.int32)
    offsets[1:] = np.cumsum(counts)
    return offsets, np.concatenate(parts) if parts else np.zeros(0, np.int32)


def two_view_pairs(seed: int = 5, n_pairs: int = 256, n_min: int = 500, n_max: int = 3000,
                   inlier_min: float = 0.3, inlier_max: float = 0.8, noise_px: float = 0.5):
    """Putative correspondences of n_pairs image pairs (the input of the apps' essential-matrix
    RANSAC): per pair a random rig (rig()), points 3..12 units in front of the first camera,
    projected into both images with N(0, noise_px^2) pixel noise, a fraction in
    [inlier_min, inlier_max] of true correspondences and the rest random positions in the right
    image.  Returns (offsets, corrs (N, 4) float32 left x, y, right x, y, K (n_pairs, 2, 3, 3),
    R (n_pairs, 3, 3), t (n_pairs, 3), inlier (N,) bool)."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(n_min, n_max + 1, n_pairs)
    offsets = np.zeros(n_pairs + 1, np.int32)
    offsets[1:] = np.cumsum(counts)
    corrs = np.empty((int(offsets[-1]), 4), np.float32)
    inl = np.zeros(int(offsets[-1]), bool)
    Ks = np.empty((n_pairs, 2, 3, 3))
    Rs = np.empty((n_pairs, 3, 3))
    ts = np.empty((n_pairs, 3))
    for p in range(n_pairs):
        K, Rot, t, _ = rig(rng, f=float(rng.uniform(900, 1500)), baseline=float(rng.uniform(0.2, 0.6)),
                           max_yaw_deg=15.0)
        n = int(counts[p])
        k = int(round(n * rng.uniform(inlier_min, inlier_max)))
        Z = rng.uniform(3.0, 12.0, n)
        uv = np.c_[rng.uniform(0, 1600, n), rng.uniform(0, 1200, n)]
        X = (np.linalg.inv(K) @ np.c_[uv, np.ones(n)].T).T * Z[:, None]
        Y = (Rot @ X.T).T + t
        q = (K @ Y.T).T
        q = q[:, :2] / q[:, 2:3]
        left = uv + rng.normal(0, noise_px, (n, 2))
        right = q + rng.normal(0, noise_px, (n, 2))
        right[k:] = np.c_[rng.uniform(0, 1600, n - k), rng.uniform(0, 1200, n - k)]
        perm = rng.permutation(n)
        b = offsets[p]
        corrs[b:b + n] = np.c_[left, right][perm].astype(np.float32)
        inl[b:b + n] = (np.arange(n) < k)[perm]
        Ks[p, 0] = K
        Ks[p, 1] = K
        Rs[p] = Rot
        ts[p] = t / np.linalg.norm(t)
    return offsets, corrs, Ks, Rs, ts, inl
