"""Literal pure-Python restatement of the reference's matching kernels for tiny cases.

Used to check the C oracle.  Each function follows V3D/CUDA/v3d_cudamatching.cu line by line
with numpy float32 scalars (one rounding per operation, like the CUDA code without
contraction):
  column scan   .cu:133-162 (per left, over rights)     row scan   .cu:164-210
  no-ratio      .cu:33-49 / :51-85                      mutual     .cu:546-551
  epipolar gate .cu:277-311                             homography .cu:313-343
"""
import numpy as np

f32 = np.float32


def score_matrix(L, R):
    """Scores[r, l] as the reference's cublasSgemm leaves them for u/512 descriptors."""
    S = R.astype(np.int64) @ L.astype(np.int64).T
    return (S.astype(np.float32) * f32(2.0 ** -18)).astype(np.float32)


def epipolar_mask(F, thr, lpos, rpos, scores):
    F1 = [f32(F[0][0]), f32(F[0][1]), f32(F[0][2])]
    F2 = [f32(F[1][0]), f32(F[1][1]), f32(F[1][2])]
    F3 = [f32(F[2][0]), f32(F[2][1]), f32(F[2][2])]
    sqr = f32(f32(thr) * f32(thr))
    out = scores.copy()
    nR, nL = scores.shape
    for col in range(nL):
        px, py = f32(lpos[col][0]), f32(lpos[col][1])
        Fpx = f32(f32(f32(F1[0] * px) + f32(F1[1] * py)) + F1[2])
        Fpy = f32(f32(f32(F2[0] * px) + f32(F2[1] * py)) + F2[2])
        Fpz = f32(f32(f32(F3[0] * px) + f32(F3[1] * py)) + F3[2])
        for row in range(nR):
            qx, qy = f32(rpos[row][0]), f32(rpos[row][1])
            Ftqx = f32(f32(f32(F1[0] * qx) + f32(F2[0] * qy)) + F3[0])
            Ftqy = f32(f32(f32(F1[1] * qx) + f32(F2[1] * qy)) + F3[1])
            num = f32(f32(f32(qx * Fpx) + f32(qy * Fpy)) + Fpz)
            num = f32(num * num)
            denom = f32(f32(f32(f32(Fpx * Fpx) + f32(Fpy * Fpy)) + f32(Ftqx * Ftqx)) + f32(Ftqy * Ftqy))
            with np.errstate(divide="ignore", invalid="ignore"):
                d = f32(num / denom)
            if d > sqr:
                out[row, col] = f32(-1e20)
    return out


def homography_mask(H, thr, lpos, rpos, scores):
    H1 = [f32(H[0][0]), f32(H[0][1]), f32(H[0][2])]
    H2 = [f32(H[1][0]), f32(H[1][1]), f32(H[1][2])]
    H3 = [f32(H[2][0]), f32(H[2][1]), f32(H[2][2])]
    sqr = f32(f32(thr) * f32(thr))
    out = scores.copy()
    nR, nL = scores.shape
    for col in range(nL):
        px, py = f32(lpos[col][0]), f32(lpos[col][1])
        x = f32(f32(f32(H1[0] * px) + f32(H1[1] * py)) + H1[2])
        y = f32(f32(f32(H2[0] * px) + f32(H2[1] * py)) + H2[2])
        z = f32(f32(f32(H3[0] * px) + f32(H3[1] * py)) + H3[2])
        with np.errstate(divide="ignore", invalid="ignore"):
            x, y = f32(x / z), f32(y / z)
        for row in range(nR):
            qx, qy = f32(rpos[row][0]), f32(rpos[row][1])
            dx, dy = f32(x - qx), f32(y - qy)
            d = f32(f32(dx * dx) + f32(dy * dy))
            if d > sqr:
                out[row, col] = f32(-1e20)
    return out


def _decide(maxVal, nextVal, argMax, minScore, minRatio):
    if minRatio < 0:
        return argMax if maxVal > f32(minScore) else -1
    nextDist = f32(max(0.001, float(f32(f32(2.0) - f32(f32(2.0) * nextVal)))))
    bestDist = f32(f32(2.0) - f32(f32(2.0) * maxVal))
    ratio = f32(bestDist / nextDist)
    return argMax if (maxVal > f32(minScore) and ratio < f32(minRatio)) else -1


def _scan(values, minScore, minRatio):
    maxVal, nextVal, argMax = f32(-1e30), f32(-1e30), -1
    for idx, val in enumerate(values):
        val = f32(val)
        gt = val > maxVal
        argMax = idx if gt else argMax
        nextVal = maxVal if gt else max(val, nextVal)
        maxVal = max(maxVal, val)
    return _decide(maxVal, nextVal, argMax, minScore, minRatio)


def match_from_scores(scores, minScore, minRatio):
    nR, nL = scores.shape
    colMax = [_scan(scores[:, l], minScore, minRatio) for l in range(nL)]
    rowMax = [_scan(scores[r, :], minScore, minRatio) for r in range(nR)]
    pairs = [(k, colMax[k]) for k in range(nL) if colMax[k] >= 0 and rowMax[colMax[k]] == k]
    return np.array(pairs, np.int32).reshape(-1, 2), np.array(colMax), np.array(rowMax)


def match(L, R, minScore, minRatio, gates=(), lpos=None, rpos=None):
    sc = score_matrix(L, R)
    for typ, M, thr in gates:
        sc = (epipolar_mask if typ == "F" else homography_mask)(M, thr, lpos, rpos, sc)
    return match_from_scores(sc, minScore, minRatio)
